// Kernels and launch templates of the explicit step, shared by the two
// translation units that compile them: nicr_step.cu (the drop-in form,
// nvcc -fmad=false, bit-identical to the reference) and nicr_step_fast.cu
// (the reciprocal form, compiled with FMA contraction). Everything here has
// internal linkage, so each unit holds its own instances of what it uses.
#pragma once
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <set>
#include <utility>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include "nicr_kernels.h"
#include "nicr_physics.h"

namespace nicr {

// Dynamic shared memory above 48 KB is opted into per kernel and per device,
// once (setting it again is harmless, skipping it on a second device is not).
static void ensure_smem_attr(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.insert({kernel, dev}).second)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

namespace {

__device__ __forceinline__ int wrapi(int v, int n) {
    v %= n;
    return v < 0 ? v + n : v;
}

// Warp + block reduction of double-double values (fixed order => deterministic).
__device__ __forceinline__ DD shfl_dd(DD v, int off) {
    DD r;
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
    return r;
}
template <int N>
__device__ void block_reduce_dd(DD (&v)[N], long long& cnt, DD* sdd, long long* scnt) {
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int w = tid >> 5, nw = (nthreads + 31) >> 5;
    // lanes of a warp are consecutive linear thread ids because blockDim.x is a multiple of 32
    for (int off = 16; off > 0; off >>= 1) {
        for (int q = 0; q < N; ++q) v[q] = dd_add(v[q], shfl_dd(v[q], off));
        cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    }
    if (lane == 0) {
        for (int q = 0; q < N; ++q) sdd[w * N + q] = v[q];
        scnt[w] = cnt;
    }
    __syncthreads();
    if (tid == 0) {
        for (int q = 0; q < N; ++q) v[q] = sdd[q];
        cnt = scnt[0];
        for (int ww = 1; ww < nw; ++ww) {
            for (int q = 0; q < N; ++q) v[q] = dd_add(v[q], sdd[ww * N + q]);
            cnt += scnt[ww];
        }
    }
}

// Tile geometry of the fused step kernel.
template <int DIM, int TA, int TB>
struct Tile {
    static constexpr int HA2 = DIM == 3 ? 2 : 0;   // row halo of the o/cr tiles
    static constexpr int HA1 = DIM == 3 ? 1 : 0;   // row halo of the phi/mu/M tiles
    static constexpr int RA2 = TA + 2 * HA2, RB2 = TB + 4;
    static constexpr int RA1 = TA + 2 * HA1, RB1 = TB + 2;
    static constexpr int S2 = RA2 * RB2, S1 = RA1 * RB1;
    // shared memory: o[4], cr[4] (halo 2); p[3] (halo 1); muO, muCr, mo, mc [2] (halo 1)
    static constexpr int SMEM_DOUBLES = 8 * S2 + 3 * S1 + 8 * S1;
    static constexpr size_t SMEM_BYTES = SMEM_DOUBLES * sizeof(double) + 64 * (5 * 16 + 8);
    static constexpr int NT = TA * TB;
    // every thread stages at most two points of each halo tile
    static_assert(2 * NT >= S2 && 2 * NT >= S1, "tile halo larger than two points per thread");
    __device__ static int i2(int a, int b) { return (a + HA2) * RB2 + (b + 2); }
    __device__ static int i1(int a, int b) { return (a + HA1) * RB1 + (b + 1); }
};

// Division by a run constant in the two arithmetic forms: FAST=false is the
// drop-in (xdiv: the correctly rounded quotient, bit-identical to a / b);
// FAST=true multiplies by RN(1/b) (within one ulp of a / b).
template <bool FAST>
__device__ __forceinline__ double fdiv(double a, const DivC& d) {
    if (FAST) return __dmul_rn(a, d.rb);
    return xdiv(a, d);
}

// Divisions of the cell arithmetic, as policies the shared arithmetic (lead
// points, cell updates) is written against. DivRun<true>: the reciprocal form.
// DivRun<false>: the exact quotient (xdiv_flag), raising `bad` for the rare
// quotients it cannot certify (subnormal, infinite or NaN, or a divisor out of
// range) instead of branching, so the march carries no branch or call per
// division; a CTA (or thread) that raised it marches again with DivExact
// before it publishes anything, so every result is still the IEEE quotient.
template <bool FAST>
struct DivRun {
    const StepParams& P;
    unsigned& bad;
    __device__ double q(double v, const DivC& d) const {
        if (FAST) return v * d.rb;   // contracted into neighbouring adds where it can
        return xdiv_flag(v, d, bad);
    }
    __device__ double dvx(double v) const { return q(v, P.v_dx); }
    __device__ double dva(double v) const { return q(v, P.v_da); }
    __device__ double dvb(double v) const { return q(v, P.v_db); }
    __device__ double dvxx(double v) const { return q(v, P.v_dxdx); }
    __device__ double dvaa(double v) const { return q(v, P.v_dada); }
    __device__ double dvbb(double v) const { return q(v, P.v_dbdb); }
    __device__ double dvt(double v) const { return q(v, P.v_dt); }
};
// exact for every numerator: xdiv, with the IEEE division (an out-of-line
// call) for numerators outside the guarded range
struct DivExact {
    const StepParams& P;
    unsigned& bad;   // unused: every result is exact
    __device__ double dvx(double v) const { return xdiv(v, P.v_dx); }
    __device__ double dva(double v) const { return xdiv(v, P.v_da); }
    __device__ double dvb(double v) const { return xdiv(v, P.v_db); }
    __device__ double dvxx(double v) const { return xdiv(v, P.v_dxdx); }
    __device__ double dvaa(double v) const { return xdiv(v, P.v_dada); }
    __device__ double dvbb(double v) const { return xdiv(v, P.v_dbdb); }
    __device__ double dvt(double v) const { return xdiv(v, P.v_dt); }
};
// The policy of a march pass: 0 the reciprocal form; 1 the drop-in form's
// first pass (exact quotients, out-of-range numerators flagged); 2 the drop-in
// form's recomputation of a CTA whose first pass raised the flag.
template <int DM> struct DivOf;
template <> struct DivOf<0> { using T = DivRun<true>; };
template <> struct DivOf<1> { using T = DivRun<false>; };
template <> struct DivOf<2> { using T = DivExact; };
// The error word a launch with parameters P reports its first failing trial to.
__device__ __forceinline__ unsigned long long* err_word(const StepParams& P, Status* st) {
    return P.err_slot < 0 ? &st->err_key : &st->slot_err[P.err_slot];
}

struct CenterVals {
    double o, cr, p, hh, muO, muCr, mo, mc;   // hh = h(p), reused by Ck
};

// SLAB instances update the plane range [P.x_lo, P.x_hi) of a slab's stored
// planes and report keys with P's offsets to P's error word; the whole-domain
// instances keep range and keys compile-time.
template <int DIM, int TA, int TB, bool FAST, bool SLAB = false>
struct StepKernel {
    using T = Tile<DIM, TA, TB>;

    // Per-thread in-plane offsets (row*pitch + col, periodic wrap applied once
    // per CTA) of the staging slots this thread fills: slot q = tid + k*NT.
    struct Offs {
        int o2[2];   // radius-2 tile points (o, cr)
        int o1[2];   // radius-1 tile points (phi)
        int gl[2];   // lead points: own cell, then the halo ring point tid (gb)
    };
    __device__ static Offs make_offs(const Grid& g, int a0, int b0) {
        Offs f;
        const int tid = threadIdx.x + TB * threadIdx.y;
        for (int k = 0; k < 2; ++k) {
            int q = tid + k * T::NT;
            f.o2[k] = -1;
            if (q < T::S2) {
                const int a = q / T::RB2 - T::HA2, b = q % T::RB2 - 2;
                f.o2[k] = (DIM == 3 ? wrapi(a0 + a, g.na) : 0) * g.pb + wrapi(b0 + b, g.nb);
            }
            f.o1[k] = -1;
            if (q < T::S1) {
                const int a = q / T::RB1 - T::HA1, b = q % T::RB1 - 1;
                f.o1[k] = (DIM == 3 ? wrapi(a0 + a, g.na) : 0) * g.pb + wrapi(b0 + b, g.nb);
            }
        }
        const int ta = DIM == 3 ? threadIdx.y : 0, tb = threadIdx.x;
        f.gl[0] = (DIM == 3 ? wrapi(a0 + ta, g.na) : 0) * g.pb + wrapi(b0 + tb, g.nb);
        f.gl[1] = -1;
        if (tid < T::S1 - T::NT) {
            int a, b;
            ring_point(tid, a, b);
            f.gl[1] = (DIM == 3 ? wrapi(a0 + a, g.na) : 0) * g.pb + wrapi(b0 + b, g.nb);
        }
        return f;
    }
    // halo ring enumeration: columns -1 and TB over all halo rows, then rows -1 and TA
    __device__ static void ring_point(int hq, int& a, int& b) {
        if (hq < 2 * T::RA1) {
            a = hq / 2 - T::HA1;
            b = (hq & 1) ? TB : -1;
        } else {
            const int r = hq - 2 * T::RA1;
            a = (r / TB) ? TA : -1;
            b = r % TB;
        }
    }

    // Loads plane xg (clamped to [0,nx-1]) of o and cr with a radius-2 halo
    // into a ring slot. The concentration inlet replaces o in plane 0 by
    // layerO before the step (enforce_legacy_layer, 3S:593-596).
    __device__ static void load_oc(const StepParams& P, const double* __restrict__ o,
                                   const double* __restrict__ cr, int xg, double* so, double* scr, const Offs& f) {
        const Grid& g = P.g;
        xg = xg < 0 ? 0 : (xg > g.nx - 1 ? g.nx - 1 : xg);
        const bool inlet = P.inlet && xg == 0;
        const long long base = (long long)xg * g.plane;
        const int tid = threadIdx.x + TB * threadIdx.y;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (f.o2[k] < 0) continue;
            const int q = tid + k * T::NT;
            const long long idx = base + f.o2[k];
            so[q] = inlet ? P.layer_o : __ldg(o + idx);
            scr[q] = __ldg(cr + idx);
        }
    }
    __device__ static void load_p(const StepParams& P, const double* __restrict__ p, int xg, double* sp,
                                  const Offs& f) {
        const Grid& g = P.g;
        xg = xg < 0 ? 0 : (xg > g.nx - 1 ? g.nx - 1 : xg);
        const long long base = (long long)xg * g.plane;
        const int tid = threadIdx.x + TB * threadIdx.y;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (f.o1[k] < 0) continue;
            sp[tid + k * T::NT] = __ldg(p + base + f.o1[k]);
        }
    }

    // Software pipelining of the staging: the loads of a later plane are issued
    // into registers before the arithmetic of the current plane and stored to
    // shared memory after it, so their latency overlaps the computation.
    struct Prefetch {
        double o[2], cr[2], p[2];
        double gbl[2];   // gb at the lead points (own cell, ring point) of the next lead plane
        double s2;       // eta_s2 at the own cell of the next update plane
    };
    // gb at the lead points of plane x (0 when grains are off)
    __device__ static void fetch_gb(const StepParams& P, const double* __restrict__ gb, int x, const Offs& f,
                                    double (&r)[2]) {
        const long long base = (long long)x * P.g.plane;
        r[0] = P.grains ? __ldg(gb + base + f.gl[0]) : 0.;
        r[1] = (P.grains && f.gl[1] >= 0) ? __ldg(gb + base + f.gl[1]) : 0.;
    }
    __device__ static void fetch(const StepParams& P, const double* __restrict__ o, const double* __restrict__ cr,
                                 const double* __restrict__ p, const double* __restrict__ gb,
                                 const double* __restrict__ s2, int xoc, int xp, int xs, bool own, const Offs& f,
                                 Prefetch& r) {
        fetch_gb(P, gb, xp, f, r.gbl);
        r.s2 = (P.phi_eta && own) ? __ldg(s2 + (long long)xs * P.g.plane + f.gl[0]) : 0.;
        const Grid& g = P.g;
        const int xo = xoc < 0 ? 0 : (xoc > g.nx - 1 ? g.nx - 1 : xoc);
        const int xq = xp < 0 ? 0 : (xp > g.nx - 1 ? g.nx - 1 : xp);
        const bool inlet = P.inlet && xo == 0;
        const long long bo = (long long)xo * g.plane, bq = (long long)xq * g.plane;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (f.o2[k] >= 0) {
                r.o[k] = inlet ? P.layer_o : __ldg(o + bo + f.o2[k]);
                r.cr[k] = __ldg(cr + bo + f.o2[k]);
            }
            if (f.o1[k] >= 0) r.p[k] = __ldg(p + bq + f.o1[k]);
        }
    }
    __device__ static void store(const Prefetch& r, double* so, double* scr, double* sp, const Offs& f) {
        const int tid = threadIdx.x + TB * threadIdx.y;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (f.o2[k] >= 0) { so[tid + k * T::NT] = r.o[k]; scr[tid + k * T::NT] = r.cr[k]; }
            if (f.o1[k] >= 0) sp[tid + k * T::NT] = r.p[k];
        }
    }

    // mu and M at tile point (a,b) of real plane x; writes the mu/M slot.
    template <class Dv>
    __device__ static CenterVals lead_core(const Dv& dv, const StepParams& k, bool o_on, const double* som,
                                           const double* so0, const double* sop, const double* scm, const double* sc0,
                                           const double* scp, const double* sp, double* smuO, double* smuCr,
                                           double* smo, double* smc, int a, int b, double gbv) {
        const int c2 = T::i2(a, b);
        const double oc = so0[c2], cc = sc0[c2];
        double lapO, lapC;
        if (DIM == 3) {
            lapO = dv.dvxx((sop[c2] - 2. * oc + som[c2]))
                 + dv.dvaa((so0[T::i2(a + 1, b)] - 2. * oc + so0[T::i2(a - 1, b)]))
                 + dv.dvbb((so0[T::i2(a, b + 1)] - 2. * oc + so0[T::i2(a, b - 1)]));
            lapC = dv.dvxx((scp[c2] - 2. * cc + scm[c2]))
                 + dv.dvaa((sc0[T::i2(a + 1, b)] - 2. * cc + sc0[T::i2(a - 1, b)]))
                 + dv.dvbb((sc0[T::i2(a, b + 1)] - 2. * cc + sc0[T::i2(a, b - 1)]));
        } else {
            lapO = dv.dvxx((sop[c2] - 2. * oc + som[c2])) + dv.dvbb((so0[T::i2(a, b + 1)] - 2. * oc + so0[T::i2(a, b - 1)]));
            lapC = dv.dvxx((scp[c2] - 2. * cc + scm[c2])) + dv.dvbb((sc0[T::i2(a, b + 1)] - 2. * cc + sc0[T::i2(a, b - 1)]));
        }
        const int c1 = T::i1(a, b);
        const double pc = sp[c1];
        const double hh = h(pc);
        CenterVals v;
        v.o = oc; v.cr = cc; v.p = pc; v.hh = hh;
        v.muO = mu_o_local(oc, cc, hh) - 2. * Phys::ko * lapO;
        v.muCr = mu_cr_local(oc, cc, hh) - 2. * Phys::kc * lapC;
        v.mo = o_on ? mobility(oc, hh, gbv, Phys::bmo, Phys::boo, k.gbm1_o) : 0.;
        v.mc = mobility(cc, hh, gbv, Phys::bmc, Phys::boc, k.gbm1_cr);
        smuO[c1] = v.muO; smuCr[c1] = v.muCr; smo[c1] = v.mo; smc[c1] = v.mc;
        return v;
    }
    // The flux divergence, phi force and Ck of the cell at (ta, tb) of plane u
    // (C: plane u, L: plane u+1, pP: phi of plane u-1, leftO/leftCr: its -X
    // face fluxes), before the trial test and the clamps.
    struct CoreOut {
        double onv, crv, pnv, rightO, rightCr, dO, dCr;
    };
    template <class Dv>
    __device__ static CoreOut cell_core(const Dv& dv, const StepParams& k, bool o_on, bool ck_legacy, bool phi_eta,
                                        const CenterVals& C, const CenterVals& L, double pP, double leftO,
                                        double leftCr, double s2u, const double* mO, const double* mC,
                                        const double* mo_, const double* mc_, const double* spu, int c1, int bp,
                                        int bm, int ap, int am) {
        CoreOut r;
        // x faces: the right face of u is the left face of u+1 (same expression)
        r.rightO = dv.dvx(-.5 * (C.mo + L.mo) * (L.muO - C.muO));
        r.rightCr = dv.dvx(-.5 * (C.mc + L.mc) * (L.muCr - C.muCr));
        double divO = 0., divCr;
        {
            const double mc0 = mc_[c1], mu0 = mC[c1];
            const double front = dv.dvb(-.5 * (mc0 + mc_[bp]) * (mC[bp] - mu0));
            const double back = dv.dvb(-.5 * (mc_[bm] + mc0) * (mu0 - mC[bm]));
            if (DIM == 3) {
                const double top = dv.dva(-.5 * (mc0 + mc_[ap]) * (mC[ap] - mu0));
                const double bottom = dv.dva(-.5 * (mc_[am] + mc0) * (mu0 - mC[am]));
                divCr = dv.dvx(leftCr - r.rightCr) + dv.dva(bottom - top) + dv.dvb(back - front);
            } else {
                divCr = dv.dvx(leftCr - r.rightCr) + dv.dvb(back - front);
            }
        }
        if (o_on) {
            const double m0 = mo_[c1], mu0 = mO[c1];
            const double front = dv.dvb(-.5 * (m0 + mo_[bp]) * (mO[bp] - mu0));
            const double back = dv.dvb(-.5 * (mo_[bm] + m0) * (mu0 - mO[bm]));
            if (DIM == 3) {
                const double top = dv.dva(-.5 * (m0 + mo_[ap]) * (mO[ap] - mu0));
                const double bottom = dv.dva(-.5 * (mo_[am] + m0) * (mu0 - mO[am]));
                divO = dv.dvx(leftO - r.rightO) + dv.dva(bottom - top) + dv.dvb(back - front);
            } else {
                divO = dv.dvx(leftO - r.rightO) + dv.dvb(back - front);
            }
        }
        const double oo = C.o, cc = C.cr, pp = C.p;
        double onv = o_on ? oo + k.dt * divO : oo;
        double crv = cc + k.dt * divCr;
        double lapP;
        if (DIM == 3)
            lapP = dv.dvxx((L.p - 2. * pp + pP)) + dv.dvaa((spu[ap] - 2. * pp + spu[am]))
                 + dv.dvbb((spu[bp] - 2. * pp + spu[bm]));
        else
            lapP = dv.dvxx((L.p - 2. * pp + pP)) + dv.dvbb((spu[bp] - 2. * pp + spu[bm]));
        const double hpv = 30. * pp * pp * (pp - 1.) * (pp - 1.);
        double fp = Phys::W * (4. * pp * pp * pp - 6. * pp * pp + 2. * pp)
                  + hpv * (foxide(oo, cc) - fmetal(oo, cc)) - 2. * Phys::kp * lapP;
        if (phi_eta) fp += grain_dphi(s2u, pp, k.eta_W, k.eta_A);
        r.pnv = pp - k.dtL * fp;
        r.dO = 0.;
        r.dCr = 0.;
        if (ck_legacy) {
            const double hn = h(r.pnv);
            r.dO = dv.dvt(-Phys::ckO * ((Phys::oxideO - onv) * hn - (Phys::oxideO - oo) * C.hh));
            r.dCr = dv.dvt(-Phys::ckCr * ((Phys::oxideCr - crv) * hn - (Phys::oxideCr - cc) * C.hh));
            onv += r.dO;
            crv += r.dCr;
        }
        r.onv = onv;
        r.crv = crv;
        return r;
    }
    // One march over the CTA's chunk with the division policy of DM (DivOf).
    // DM 1 returns true, without publishing its failure keys or budget
    // partials, when a numerator of the chunk left the guarded range.
    template <int DM>
    __device__ static bool run_body(const StepParams& P, const double* __restrict__ o, const double* __restrict__ cr,
                                    const double* __restrict__ p, const double* __restrict__ gb,
                                    const double* __restrict__ s2, double* __restrict__ on,
                                    double* __restrict__ crn, double* __restrict__ pn,
                                    StepPartial* __restrict__ partials, Status* st, int bx, int by, int bz, int blin) {
        extern __shared__ __align__(16) double smem[];
        double* so = smem;                 // 4 slots x S2
        double* scr = so + 4 * T::S2;      // 4 slots x S2
        double* sp = scr + 4 * T::S2;      // 3 slots x S1
        double* smuO = sp + 3 * T::S1;     // 2 slots x S1
        double* smuCr = smuO + 2 * T::S1;
        double* smo = smuCr + 2 * T::S1;
        double* smc = smo + 2 * T::S1;
        DD* sdd = reinterpret_cast<DD*>(smc + 2 * T::S1);
        long long* scnt = reinterpret_cast<long long*>(sdd + 32 * 5);

        const Grid& g = P.g;
        const int ta = DIM == 3 ? threadIdx.y : 0, tb = threadIdx.x;
        const int a0 = DIM == 3 ? by * TA : 0, b0 = bx * TB;
        const int i0 = (SLAB ? P.x_lo : 0) + bz * P.xchunk;
        const int i1 = min(SLAB ? P.x_hi : g.nx, i0 + P.xchunk);
        const int row = a0 + ta, col = b0 + tb;
        const bool active = (DIM == 3 ? row < g.na : true) && col < g.nb;
        const Offs offs = make_offs(g, a0, b0);

        DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};  // ckO ckCr clipO clipCr bcO
        long long clipped = 0;
        unsigned long long errkey = ERR_NONE;

        if (st->failed) return false;  // a previous step of this batch was rejected
        unsigned bad = 0;
        const typename DivOf<DM>::T dv{P, bad};

        auto slot3 = [](int w) { return ((w % 3) + 3) % 3; };
        // o/cr ring of 4 planes: the plane staged at the top of an iteration
        // (x+2) never overlaps the window x-1..x+1 that slower warps may still
        // be reading in lead(x), so one barrier per plane suffices
        auto oslot = [&](int w) { return so + (w & 3) * T::S2; };
        auto cslot = [&](int w) { return scr + (w & 3) * T::S2; };
        auto pslot = [&](int x) { return sp + slot3(x) * T::S1; };

        // Computes the lead plane x (real plane) over the tile + radius-1 halo.
        auto lead = [&](int x, const double (&gbl)[2]) -> CenterVals {
            const double *som = oslot(x - 1), *so0 = oslot(x), *sop = oslot(x + 1);
            const double *scm = cslot(x - 1), *sc0 = cslot(x), *scp = cslot(x + 1);
            const double* spx = pslot(x);
            double* mO = smuO + (x & 1) * T::S1;
            double* mC = smuCr + (x & 1) * T::S1;
            double* mo_ = smo + (x & 1) * T::S1;
            double* mc_ = smc + (x & 1) * T::S1;
            CenterVals own = lead_core(dv, P, P.o_on != 0, som, so0, sop, scm, sc0, scp, spx, mO, mC, mo_, mc_, ta,
                                       tb, gbl[0]);
            // halo ring points: one per thread for the first S1-NT threads
            static_assert(T::S1 - T::NT <= T::NT, "ring larger than the CTA");
            const int tid = threadIdx.x + TB * threadIdx.y;
            if (offs.gl[1] >= 0) {
                int a, b;
                ring_point(tid, a, b);
                lead_core(dv, P, P.o_on != 0, som, so0, sop, scm, sc0, scp, spx, mO, mC, mo_, mc_, a, b, gbl[1]);
            }
            return own;
        };

        CenterVals C, L;
        double pP, FxO, FxCr;
        // ---- prologue: centre values of the first update plane and its left x-face flux
        if (i0 == 0) {
            load_oc(P, o, cr, -1, oslot(-1), cslot(-1), offs);
            load_oc(P, o, cr, 0, oslot(0), cslot(0), offs);
            load_oc(P, o, cr, 1, oslot(1), cslot(1), offs);
            load_p(P, p, 0, pslot(0), offs);
            double gb0[2];
            fetch_gb(P, gb, 0, offs, gb0);
            __syncthreads();
            C = lead(0, gb0);
            __syncthreads();
            // ghost plane -1: copies of plane 0 (3S:187, 3S:613-615, 3S:616-619)
            const double muOg = (P.bc == 1 && P.o_on) ? 2. * P.mu_res - C.muO : C.muO;
            FxO = dv.dvx(-.5 * (C.mo + C.mo) * (C.muO - muOg));
            FxCr = dv.dvx(-.5 * (C.mc + C.mc) * (C.muCr - C.muCr));
            pP = C.p;
        } else {
            load_oc(P, o, cr, i0 - 2, oslot(i0 - 2), cslot(i0 - 2), offs);
            load_oc(P, o, cr, i0 - 1, oslot(i0 - 1), cslot(i0 - 1), offs);
            load_oc(P, o, cr, i0, oslot(i0), cslot(i0), offs);
            load_p(P, p, i0 - 1, pslot(i0 - 1), offs);
            double gbm[2];
            fetch_gb(P, gb, i0 - 1, offs, gbm);
            __syncthreads();
            const CenterVals Pv = lead(i0 - 1, gbm);
            load_oc(P, o, cr, i0 + 1, oslot(i0 + 1), cslot(i0 + 1), offs);
            load_p(P, p, i0, pslot(i0), offs);
            double gb0[2];
            fetch_gb(P, gb, i0, offs, gb0);
            __syncthreads();
            C = lead(i0, gb0);
            __syncthreads();
            FxO = dv.dvx(-.5 * (Pv.mo + C.mo) * (C.muO - Pv.muO));
            FxCr = dv.dvx(-.5 * (Pv.mc + C.mc) * (C.muCr - Pv.muCr));
            pP = Pv.p;
        }

        double s2u = (P.phi_eta && active) ? __ldg(s2 + (long long)i0 * g.plane + offs.gl[0]) : 0.;
        Prefetch pf;
        if (i0 + 1 <= g.nx - 1) fetch(P, o, cr, p, gb, s2, i0 + 2, i0 + 1, i0 + 1, active, offs, pf);
        for (int u = i0; u < i1; ++u) {
            const int x = u + 1;
            double s2n = 0.;
            if (x <= g.nx - 1) {
                // one barrier per plane: it orders this plane's staging before
                // lead(x), and the previous update(u-1) (which read the mu/M
                // slot lead(x) now overwrites) before lead(x)
                store(pf, oslot(x + 1), cslot(x + 1), pslot(x), offs);
                const double gbl[2] = {pf.gbl[0], pf.gbl[1]};
                s2n = pf.s2;
                __syncthreads();
                if (x + 1 <= g.nx - 1 && u + 1 < i1)
                    fetch(P, o, cr, p, gb, s2, x + 2, x + 1, x + 1, active, offs, pf);
                L = lead(x, gbl);
            } else {
                L = C;  // ghost plane nx: Neumann copy of plane nx-1 (mu and M copied too)
                // no staging in this iteration, but update(nx-1) reads the mu/M
                // that lead(nx-1) of other warps wrote in the previous one
                __syncthreads();
            }
            if (active) {
                const double* mO = smuO + (u & 1) * T::S1;
                const double* mC = smuCr + (u & 1) * T::S1;
                const double* mo_ = smo + (u & 1) * T::S1;
                const double* mc_ = smc + (u & 1) * T::S1;
                const double* spu = pslot(u);
                const int c1 = T::i1(ta, tb);
                const int bp = T::i1(ta, tb + 1), bm = T::i1(ta, tb - 1);
                const int ap = T::i1(ta + 1, tb), am = T::i1(ta - 1, tb);
                const long long gidx = (long long)u * g.plane + (long long)row * g.pb + col;
                const long long cell = ((long long)u * g.na + row) * g.nb + col + (SLAB ? P.cell_off : 0);  // reference loop order

                double leftO = FxO;
                if (u == 0 && P.bc == 1) {
                    // left_flux (3S:621-628): surface-mobility face closure for bc=mu
                    double lf = 0.;
                    if (P.o_on) {
                        const double gb0 = P.grains ? __ldg(gb + gidx) : 0.;
                        const double mf = mobility(P.surface_c_ref, h(C.p), gb0, Phys::bmo, Phys::boo, P.gbm1_o);
                        lf = dv.dvx(2. * mf * (P.mu_res - C.muO));
                    }
                    leftO = lf;
                    acc[4] = dd_add(acc[4], dv.dvx(P.dt * lf));
                }
                if (u == 0 && P.inlet) acc[4] = dd_add(acc[4], P.layer_o - __ldg(o + gidx));

                // fluxes, phi force and Ck (3S:761-811); the trial test and the
                // clamps below without data-dependent branches (so the scheduler
                // sees one block); the rare bookkeeping (budget terms of changed
                // cells, failure keys) is one branch after the stores
                const CoreOut R = cell_core(dv, P, P.o_on != 0, P.ck == 0, P.phi_eta != 0, C, L, pP, leftO, FxCr,
                                            s2u, mO, mC, mo_, mc_, spu, c1, bp, bm, ap, am);
                double onv = R.onv, crv = R.crv, pnv = R.pnv;
                const double dO = R.dO, dCr = R.dCr, rightO = R.rightO, rightCr = R.rightCr;
                const bool nonfinite = !isfinite(onv) || !isfinite(crv) || !isfinite(pnv);
                double clO = 0., clCr = 0.;
                bool outside = false;
                if (P.bounds == 1) {
                    const double oc = sclamp(onv, 0., 1.), ccr = sclamp(crv, 0., 1.);
                    if (!nonfinite) {
                        clO = oc - onv;
                        clCr = ccr - crv;
                        clipped += (oc != onv || ccr != crv) ? 1 : 0;
                        onv = oc;
                        crv = ccr;
                        pnv = pnv > .99999 ? 1. : pnv;
                        pnv = pnv < 1.e-5 ? 0. : pnv;
                    }
                } else {
                    outside = !nonfinite && (onv < -1.e-12 || crv < -1.e-12 || onv + crv > 1. + 1.e-12 ||
                                             pnv < -1.e-12 || pnv > 1. + 1.e-12);
                }
                on[gidx] = onv; crn[gidx] = crv; pn[gidx] = pnv;
                FxO = rightO; FxCr = rightCr;
                if (nonfinite || outside || dO != 0. || dCr != 0. || clO != 0. || clCr != 0.) {
                    if (nonfinite || outside) errkey = min(errkey, (unsigned long long)cell * 4ull + (nonfinite ? 0ull : 1ull));
                    // adding +-0 to a normalised double-double leaves it unchanged,
                    // so zero increments (metal cells: h(pn) == h(p) == 0) are skipped
                    if (dO != 0.) acc[0] = dd_add(acc[0], dO);
                    if (dCr != 0.) acc[1] = dd_add(acc[1], dCr);
                    if (clO != 0.) acc[2] = dd_add(acc[2], clO);
                    if (clCr != 0.) acc[3] = dd_add(acc[3], clCr);
                }
            }
            pP = C.p;
            C = L;
            s2u = s2n;
        }
        if (DM == 1 && __syncthreads_or(bad != 0)) return true;
        if (errkey != ERR_NONE) atomicMin(SLAB ? err_word(P, st) : &st->err_key, errkey);
        block_reduce_dd<5>(acc, clipped, sdd, scnt);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            StepPartial& out = partials[blin];
            for (int q = 0; q < 5; ++q) { out.s[q][0] = acc[q].hi; out.s[q][1] = acc[q].lo; }
            out.clipped = clipped;
            out.redo = 0;
        }
        return false;
    }

    // One CTA's chunk. In the drop-in form a chunk whose numerators left the
    // guarded range is marched again with every quotient exact (IEEE division
    // for those), rewriting its trial values, before keys and partials are
    // published: here (DEFER false), or by k_step_redo after the launch
    // (DEFER true: the CTA only marks its partial slot), which keeps the
    // second march and its division calls out of the hot kernel.
    template <bool DEFER = false>
    __device__ static void run(const StepParams& P, const double* __restrict__ o, const double* __restrict__ cr,
                               const double* __restrict__ p, const double* __restrict__ gb,
                               const double* __restrict__ s2, double* __restrict__ on,
                               double* __restrict__ crn, double* __restrict__ pn,
                               StepPartial* __restrict__ partials, Status* st, int bx, int by, int bz, int blin) {
        if (FAST) {
            run_body<0>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, bx, by, bz, blin);
        } else if (run_body<1>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, bx, by, bz, blin)) {
            if (DEFER) {
                if (threadIdx.x == 0 && threadIdx.y == 0) partials[blin].redo = 1;
            } else {
                __syncthreads();
                run_body<2>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, bx, by, bz, blin);
            }
        }
    }
};

template <int DIM, int TA, int TB, int MINB, bool FAST, bool SLAB = false>
__global__ void __launch_bounds__(TA * TB, MINB)
k_step_main(const StepParams P, const double* __restrict__ o, const double* __restrict__ cr,
            const double* __restrict__ p, const double* __restrict__ gb, const double* __restrict__ s2,
            double* __restrict__ on, double* __restrict__ crn, double* __restrict__ pn,
            StepPartial* __restrict__ partials, Status* st) {
    StepKernel<DIM, TA, TB, FAST, SLAB>::template run<true>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, blockIdx.x,
                                                            blockIdx.y, blockIdx.z,
                                                            blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
}

// The drop-in form's recomputation of the chunks k_step_main marked (numerators
// outside the exact-division range, which its march only flags): each CTA
// takes marked chunks of the step grid (gx x gy x gz CTAs) in turn and marches
// them with every quotient exact, rewriting trial values, key and partials.
template <int DIM, int TA, int TB, bool SLAB = false>
__global__ void __launch_bounds__(TA * TB, 1)
k_step_redo(const StepParams P, const double* __restrict__ o, const double* __restrict__ cr,
            const double* __restrict__ p, const double* __restrict__ gb, const double* __restrict__ s2,
            double* __restrict__ on, double* __restrict__ crn, double* __restrict__ pn,
            StepPartial* __restrict__ partials, Status* st, int gx, int gy, int nblocks) {
    for (int blin = blockIdx.x; blin < nblocks; blin += gridDim.x) {
        if (!partials[blin].redo) continue;   // the same word for the whole CTA
        __syncthreads();                      // the previous chunk's shared-memory reads are done
        StepKernel<DIM, TA, TB, false, SLAB>::template run_body<2>(P, o, cr, p, gb, s2, on, crn, pn, partials, st,
                                                                   blin % gx, (blin / gx) % gy, blin / (gx * gy),
                                                                   blin);
    }
}

constexpr int TA3 = 8, TB3 = 32;    // 3D tile: 8 rows x 32 columns, 256 threads
constexpr int TA2 = 1, TB2 = 128;   // 2D tile: 128 columns

template <int DIM, int TA, int TB>
dim3 step_grid(const StepParams& P) {
    const Grid& g = P.g;
    return dim3((g.nb + TB - 1) / TB, DIM == 3 ? (g.na + TA - 1) / TA : 1, (P.x_hi - P.x_lo + P.xchunk - 1) / P.xchunk);
}

// eta_trial (3S:514-526): v = eta - (dt*L_eta)*(deta - K*lap(eta)); must lie in
// [-1e-12, 1+1e-12]. Writes the trial and the mask of the trial values (the
// next step's gb and eta_s2, identical to rebuild_eta_mask on them).
template <int DIM, int DM>
__device__ __forceinline__ unsigned eta_cell_pass(const StepParams& P, int neta, const double* __restrict__ eta,
                                         const double* __restrict__ s2, const double* __restrict__ p,
                                         double* __restrict__ eta_next, double* __restrict__ gb_next,
                                         double* __restrict__ s2_next, int x, int row, int col,
                                         unsigned long long& errkey) {
    const Grid& g = P.g;
    unsigned dbad = 0;
    const typename DivOf<DM>::T dv{P, dbad};
    const long long idx = (long long)x * g.plane + (long long)row * g.pb + col;
    const long long cell = ((long long)x * g.na + row) * g.nb + col + P.cell_off;
    const long long ixm = x > 0 ? idx - g.plane : idx, ixp = x < g.nx - 1 ? idx + g.plane : idx;
    const long long rbase = (long long)x * g.plane;
    const long long ibm = rbase + (long long)row * g.pb + (col == 0 ? g.nb - 1 : col - 1);
    const long long ibp = rbase + (long long)row * g.pb + (col == g.nb - 1 ? 0 : col + 1);
    long long iam = idx, iap = idx;
    if (DIM == 3) {
        iam = rbase + (long long)(row == 0 ? g.na - 1 : row - 1) * g.pb + col;
        iap = rbase + (long long)(row == g.na - 1 ? 0 : row + 1) * g.pb + col;
    }
    const double S = __ldg(s2 + idx), phi = __ldg(p + idx);
    double Sn = 0., pairs = 0.;
    int first_bad = -1;   // the first field failing the range test
    for (int q = 0; q < neta; ++q) {
        const double* e = eta + (long long)q * g.nstore;
        const double ec = __ldg(e + idx);
        double lap;
        if (DIM == 3)
            lap = dv.dvxx((__ldg(e + ixp) - 2. * ec + __ldg(e + ixm))) + dv.dvaa((__ldg(e + iap) - 2. * ec + __ldg(e + iam)))
                + dv.dvbb((__ldg(e + ibp) - 2. * ec + __ldg(e + ibm)));
        else
            lap = dv.dvxx((__ldg(e + ixp) - 2. * ec + __ldg(e + ixm))) + dv.dvbb((__ldg(e + ibp) - 2. * ec + __ldg(e + ibm)));
        const double force = grain_deta(ec, S, phi, P.eta_W, P.eta_A) - P.eta_K * lap;
        const double v = ec - P.dt_etaL * force;
        const bool fail = !(v >= -1.e-12 && v <= 1. + 1.e-12);   // NaN fails both comparisons
        first_bad = (fail && first_bad < 0) ? q : first_bad;
        eta_next[(long long)q * g.nstore + idx] = v;
        const double sq = v * v;
        pairs += Sn * sq;
        Sn += sq;
    }
    // keyed once per cell: the first failing field in reference order
    if (first_bad >= 0)
        errkey = min(errkey, ERR_ETA_BASE + (unsigned long long)first_bad * (unsigned long long)P.key_ncells +
                                 (unsigned long long)cell);
    s2_next[idx] = Sn;
    gb_next[idx] = P.eta_scale * smin(1., 16. * pairs);
    return dbad;
}
// The cell's eta update with the division policy of the form; in the drop-in
// form a cell whose numerators left the exact-division range is recomputed
// with every quotient exact (its values rewritten, its key taken from the
// recomputation).
template <int DIM, bool FAST>
__device__ __forceinline__ void eta_cell(const StepParams& P, int neta, const double* __restrict__ eta,
                                         const double* __restrict__ s2, const double* __restrict__ p,
                                         double* __restrict__ eta_next, double* __restrict__ gb_next,
                                         double* __restrict__ s2_next, int x, int row, int col,
                                         unsigned long long& errkey) {
    if (FAST) {
        eta_cell_pass<DIM, 0>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, x, row, col, errkey);
        return;
    }
    unsigned long long k = ERR_NONE;
    if (eta_cell_pass<DIM, 1>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, x, row, col, k)) {
        k = ERR_NONE;
        eta_cell_pass<DIM, 2>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, x, row, col, k);
    }
    errkey = min(errkey, k);
}

// Bounds for 5 CTAs/SM (<= 51 registers, no spills): the load-latency-bound
// per-cell kernel measured 1.13 ms vs 1.29 ms unbounded (62 registers, 4/SM)
// at 256^3 with 8 fields; 6/SM spills (1.27 ms).
template <int DIM, bool FAST>
__global__ void __launch_bounds__(256, 5) k_eta_update(const StepParams P, int neta, const double* __restrict__ eta,
                             const double* __restrict__ s2, const double* __restrict__ p,
                             double* __restrict__ eta_next, double* __restrict__ gb_next,
                             double* __restrict__ s2_next, Status* st) {
    if (st->failed) return;
    const Grid& g = P.g;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = DIM == 3 ? blockIdx.y * blockDim.y + threadIdx.y : 0;
    if (col >= g.nb || row >= g.na) return;
    unsigned long long errkey = ERR_NONE;
    eta_cell<DIM, FAST>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, P.x_lo + blockIdx.z, row, col, errkey);
    if (errkey != ERR_NONE) atomicMin(err_word(P, st), errkey);
}

// X-marching form of the eta update for a compile-time number of fields N:
// each thread owns one (row, col) column of a chunk of planes and keeps
// eta(x-1), eta(x), eta(x+1) of its column in registers, so each field value
// is read from HBM once; the four in-plane neighbours come from L1 (they are
// the neighbouring threads' own loads). All N loads of the next plane are
// issued before the arithmetic of the current plane.
// NCAP is the register capacity; the first n <= NCAP fields are updated (the
// stand-alone kernel instantiates NCAP = n, so the guards fold away). SLAB
// instances take the plane range and key offsets from P; the whole-domain
// instances keep them compile-time (the runtime range cost this kernel's
// schedule 85% at 128 registers).
// One march of a thread's column with the division policy of DM (DivOf);
// returns the flag of numerators outside the exact-division range (DM 1).
template <int DIM, int DM, int NCAP, bool SLAB>
__device__ __forceinline__ unsigned eta_march_pass(const StepParams& P, int n, const double* __restrict__ eta,
                                                   const double* __restrict__ p, double* __restrict__ eta_next,
                                                   double* __restrict__ gb_next, double* __restrict__ s2_next,
                                                   int row, int col, int i0, int i1, unsigned long long& errkey) {
    const Grid& g = P.g;
    unsigned dbad = 0;
    const typename DivOf<DM>::T dv{P, dbad};
    const long long rc = (long long)row * g.pb + col;
    const long long cbm = (long long)row * g.pb + (col == 0 ? g.nb - 1 : col - 1);
    const long long cbp = (long long)row * g.pb + (col == g.nb - 1 ? 0 : col + 1);
    long long cam = rc, cap = rc;
    if (DIM == 3) {
        cam = (long long)(row == 0 ? g.na - 1 : row - 1) * g.pb + col;
        cap = (long long)(row == g.na - 1 ? 0 : row + 1) * g.pb + col;
    }
    double ep[NCAP], ec[NCAP], en[NCAP];
    {
        const long long bm = (long long)(i0 > 0 ? i0 - 1 : 0) * g.plane, b0 = (long long)i0 * g.plane;
#pragma unroll
        for (int q = 0; q < NCAP; ++q) {
            if (q < n) {
                ep[q] = __ldg(eta + (long long)q * g.nstore + bm + rc);
                ec[q] = __ldg(eta + (long long)q * g.nstore + b0 + rc);
            }
        }
    }
    for (int x = i0; x < i1; ++x) {
        const long long base = (long long)x * g.plane;
        const long long bnext = (long long)(x < g.nx - 1 ? x + 1 : x) * g.plane;
#pragma unroll
        for (int q = 0; q < NCAP; ++q)
            if (q < n) en[q] = __ldg(eta + (long long)q * g.nstore + bnext + rc);
        const double phi = __ldg(p + base + rc);
        double S = 0.;
#pragma unroll
        for (int q = 0; q < NCAP; ++q)
            if (q < n) S += ec[q] * ec[q];
        const long long cell = ((long long)x * g.na + row) * g.nb + col + (SLAB ? P.cell_off : 0);
        double Sn = 0., pairs = 0.;
        unsigned bad = 0;
#pragma unroll
        for (int q = 0; q < NCAP; ++q) {
            if (q >= n) break;
            const double* e = eta + (long long)q * g.nstore + base;
            const double c0 = ec[q];
            double lap;
            if (DIM == 3)
                lap = dv.dvxx((en[q] - 2. * c0 + ep[q])) + dv.dvaa((__ldg(e + cap) - 2. * c0 + __ldg(e + cam)))
                    + dv.dvbb((__ldg(e + cbp) - 2. * c0 + __ldg(e + cbm)));
            else
                lap = dv.dvxx((en[q] - 2. * c0 + ep[q])) + dv.dvbb((__ldg(e + cbp) - 2. * c0 + __ldg(e + cbm)));
            const double force = grain_deta(c0, S, phi, P.eta_W, P.eta_A) - P.eta_K * lap;
            const double v = c0 - P.dt_etaL * force;
            bad |= !(v >= -1.e-12 && v <= 1. + 1.e-12) ? (1u << q) : 0u;   // NaN fails both comparisons
            eta_next[(long long)q * g.nstore + base + rc] = v;
            const double sq = v * v;
            pairs += Sn * sq;
            Sn += sq;
        }
        // fields failing the range test, keyed once (the first in reference order)
        if (bad)
            errkey = min(errkey, ERR_ETA_BASE + (unsigned long long)(__ffs(bad) - 1) *
                                     (unsigned long long)(SLAB ? P.key_ncells : g.ncells) + (unsigned long long)cell);
        s2_next[base + rc] = Sn;
        gb_next[base + rc] = P.eta_scale * smin(1., 16. * pairs);
#pragma unroll
        for (int q = 0; q < NCAP; ++q)
            if (q < n) { ep[q] = ec[q]; ec[q] = en[q]; }
    }
    return dbad;
}

// X-marching form of the eta update for a compile-time number of fields N:
// each thread owns one (row, col) column of a chunk of planes and keeps
// eta(x-1), eta(x), eta(x+1) of its column in registers, so each field value
// is read from HBM once; the four in-plane neighbours come from L1 (they are
// the neighbouring threads' own loads). All N loads of the next plane are
// issued before the arithmetic of the current plane.
// NCAP is the register capacity; the first n <= NCAP fields are updated (the
// stand-alone kernel instantiates NCAP = n, so the guards fold away). SLAB
// instances take the plane range and key offsets from P; the whole-domain
// instances keep them compile-time (the runtime range cost this kernel's
// schedule 85% at 128 registers). In the drop-in form a column whose
// numerators left the exact-division range is marched again with every
// quotient exact before its key is merged (its trial values rewritten).
template <int DIM, bool FAST, int NCAP, bool SLAB = false>
__device__ __forceinline__ void eta_march_body(const StepParams& P, int n, const double* __restrict__ eta,
                                               const double* __restrict__ p, double* __restrict__ eta_next,
                                               double* __restrict__ gb_next, double* __restrict__ s2_next,
                                               Status* st, int bx, int by, int bz) {
    if (st->failed) return;
    const Grid& g = P.g;
    const int col = bx * blockDim.x + threadIdx.x;
    const int row = DIM == 3 ? by * blockDim.y + threadIdx.y : 0;
    if (col >= g.nb || row >= g.na) return;
    const int i0 = (SLAB ? P.x_lo : 0) + bz * P.xchunk, i1 = min(SLAB ? P.x_hi : g.nx, i0 + P.xchunk);
    unsigned long long errkey = ERR_NONE;
    if (FAST) {
        eta_march_pass<DIM, 0, NCAP, SLAB>(P, n, eta, p, eta_next, gb_next, s2_next, row, col, i0, i1, errkey);
    } else if (eta_march_pass<DIM, 1, NCAP, SLAB>(P, n, eta, p, eta_next, gb_next, s2_next, row, col, i0, i1,
                                                   errkey)) {
        errkey = ERR_NONE;
        eta_march_pass<DIM, 2, NCAP, SLAB>(P, n, eta, p, eta_next, gb_next, s2_next, row, col, i0, i1, errkey);
    }
    if (errkey != ERR_NONE) atomicMin(SLAB ? err_word(P, st) : &st->err_key, errkey);
}

// 2 CTAs/SM stated in the bounds: the register count stays <= 128 either way,
// but the schedule compiled for it measured 15% faster on B200 (0.58 vs 0.69
// ms at 256^3 with 8 fields, same box); bounds for 3 CTAs/SM spill and lose.
template <int DIM, bool FAST, int N, bool SLAB = false>
__global__ void __launch_bounds__(256, 2)
k_eta_march(const StepParams P, const double* __restrict__ eta, const double* __restrict__ p,
            double* __restrict__ eta_next, double* __restrict__ gb_next, double* __restrict__ s2_next, Status* st) {
    eta_march_body<DIM, FAST, N, SLAB>(P, N, eta, p, eta_next, gb_next, s2_next, st, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <int DIM, bool FAST, int N>
static void launch_eta_march(const StepParams& P, const double* eta, const double* p, double* eta_next,
                             double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    const Grid& g = P.g;
    if (DIM == 3) {
        const dim3 grid((g.nb + 31) / 32, (g.na + 7) / 8, (P.x_hi - P.x_lo + P.xchunk - 1) / P.xchunk);
        if (P.err_slot >= 0)   // an X slab (3D only)
            k_eta_march<3, FAST, N, true><<<grid, dim3(32, 8), 0, stream>>>(P, eta, p, eta_next, gb_next, s2_next, st);
        else
            k_eta_march<3, FAST, N><<<grid, dim3(32, 8), 0, stream>>>(P, eta, p, eta_next, gb_next, s2_next, st);
    } else {
        const dim3 grid((g.nb + 127) / 128, 1, (g.nx + P.xchunk - 1) / P.xchunk);
        k_eta_march<2, FAST, N><<<grid, dim3(128, 1), 0, stream>>>(P, eta, p, eta_next, gb_next, s2_next, st);
    }
}

// Horizontal fusion of the step kernel and the eta march (3D): within a step
// the two are independent (the step kernel reads o, cr, phi, gb, eta_s2 and
// writes the trial o, cr, phi; the eta update reads eta and the current phi
// and writes the next eta, gb, eta_s2), and the step kernel is bound by FP64
// issue while the march waits on HBM. Each CTA draws a ticket and takes the
// step tile or the eta column block the ticket names; the tickets alternate
// between the two kinds while both last, so the SMs run both kinds at once
// and their pipes overlap. The CTAs compute what the separate kernels compute
// (the same bodies; step partial sums at the step kernel's block index).
// Opt-in (NICR_FUSED=1): at 256^3 with 8 fields it measured 1.122 ms per step
// against 1.129 ms for the two launches. Both kernels hold 2 CTAs/SM at 128
// registers and each is bound by the latency its own warps hide; an SM that
// runs one CTA of each gives each kind half the warps, which costs about what
// the overlap gains.
struct FusedStep {
    int n_step, n_eta;     // CTAs of each kind
    int gx_s, gy_s;        // step grid (x, y; z = X chunks)
    int gx_e, gy_e;        // eta march grid (x, y; z = X chunks)
    unsigned* ticket;      // zero at launch
};
template <bool FAST, int N>
__global__ void __launch_bounds__(TA3 * TB3, 2)
k_step_eta(const StepParams P, const FusedStep F, const double* __restrict__ o, const double* __restrict__ cr,
           const double* __restrict__ p, const double* __restrict__ gb, const double* __restrict__ s2,
           double* __restrict__ on, double* __restrict__ crn, double* __restrict__ pn,
           StepPartial* __restrict__ partials, const double* __restrict__ eta, double* __restrict__ eta_next,
           double* __restrict__ gb_next, double* __restrict__ s2_next, Status* st) {
    __shared__ int s_ticket;
    if (threadIdx.x == 0 && threadIdx.y == 0) s_ticket = (int)atomicAdd(F.ticket, 1u);
    __syncthreads();
    const int t = s_ticket, pairs = min(F.n_step, F.n_eta);
    int role, idx;
    if (t < 2 * pairs) {
        role = t & 1;
        idx = t >> 1;
    } else {
        role = F.n_step > F.n_eta ? 0 : 1;
        idx = pairs + (t - 2 * pairs);
    }
    if (role == 0) {
        const int bx = idx % F.gx_s, r = idx / F.gx_s;
        StepKernel<3, TA3, TB3, FAST>::run(P, o, cr, p, gb, s2, on, crn, pn, partials, st, bx, r % F.gy_s,
                                           r / F.gy_s, idx);
    } else {
        const int bx = idx % F.gx_e, r = idx / F.gx_e;
        eta_march_body<3, FAST, N>(P, N, eta, p, eta_next, gb_next, s2_next, st, bx, r % F.gy_e, r / F.gy_e);
    }
}

template <bool FAST, int N>
static void launch_step_eta_n(const StepParams& P, const double* o, const double* cr, const double* p,
                              const double* gb, const double* s2, double* on, double* crn, double* pn,
                              StepPartial* partials, const double* eta, double* eta_next, double* gb_next,
                              double* s2_next, unsigned* ticket, Status* st, cudaStream_t stream, int* nblocks_out) {
    using T = Tile<3, TA3, TB3>;
    const Grid& g = P.g;
    const dim3 gs = step_grid<3, TA3, TB3>(P);
    const dim3 ge((g.nb + 31) / 32, (g.na + 7) / 8, (P.x_hi - P.x_lo + P.xchunk - 1) / P.xchunk);
    FusedStep F;
    F.gx_s = (int)gs.x; F.gy_s = (int)gs.y; F.n_step = (int)(gs.x * gs.y * gs.z);
    F.gx_e = (int)ge.x; F.gy_e = (int)ge.y; F.n_eta = (int)(ge.x * ge.y * ge.z);
    F.ticket = ticket;
    ensure_smem_attr((const void*)k_step_eta<FAST, N>, (int)T::SMEM_BYTES);
    cudaMemsetAsync(ticket, 0, sizeof(unsigned), stream);
    k_step_eta<FAST, N><<<F.n_step + F.n_eta, dim3(TB3, TA3), T::SMEM_BYTES, stream>>>(
        P, F, o, cr, p, gb, s2, on, crn, pn, partials, eta, eta_next, gb_next, s2_next, st);
    if (nblocks_out) *nblocks_out = F.n_step;
}

template <bool FAST>
static void step_eta_prepare(int neta) {
    using T = Tile<3, TA3, TB3>;
    switch (neta) {
#define NICR_FUSED_PREP(n) \
    case n: ensure_smem_attr((const void*)k_step_eta<FAST, n>, (int)T::SMEM_BYTES); break;
        NICR_FUSED_PREP(1) NICR_FUSED_PREP(2) NICR_FUSED_PREP(3) NICR_FUSED_PREP(4) NICR_FUSED_PREP(5)
        NICR_FUSED_PREP(6) NICR_FUSED_PREP(7) NICR_FUSED_PREP(8) NICR_FUSED_PREP(9) NICR_FUSED_PREP(10)
        NICR_FUSED_PREP(11) NICR_FUSED_PREP(12) NICR_FUSED_PREP(13) NICR_FUSED_PREP(14) NICR_FUSED_PREP(15)
        NICR_FUSED_PREP(16)
#undef NICR_FUSED_PREP
        default: break;
    }
}

template <bool FAST>
static bool launch_step_eta_form(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                                 const double* gb, const double* s2, double* on, double* crn, double* pn,
                                 StepPartial* partials, const double* eta, double* eta_next, double* gb_next,
                                 double* s2_next, unsigned* ticket, Status* st, cudaStream_t stream,
                                 int* nblocks_out) {
    if (P.g.dim != 3 || P.err_slot >= 0) return false;
    switch (neta) {
#define NICR_FUSED_CASE(n)                                                                                   \
    case n:                                                                                                  \
        launch_step_eta_n<FAST, n>(P, o, cr, p, gb, s2, on, crn, pn, partials, eta, eta_next, gb_next, s2_next, \
                                   ticket, st, stream, nblocks_out);                                         \
        return true;
        NICR_FUSED_CASE(1) NICR_FUSED_CASE(2) NICR_FUSED_CASE(3) NICR_FUSED_CASE(4) NICR_FUSED_CASE(5)
        NICR_FUSED_CASE(6) NICR_FUSED_CASE(7) NICR_FUSED_CASE(8) NICR_FUSED_CASE(9) NICR_FUSED_CASE(10)
        NICR_FUSED_CASE(11) NICR_FUSED_CASE(12) NICR_FUSED_CASE(13) NICR_FUSED_CASE(14) NICR_FUSED_CASE(15)
        NICR_FUSED_CASE(16)
#undef NICR_FUSED_CASE
        default: return false;
    }
}

// Dispatch to the compile-time field counts 1..16; false when N is larger.
template <int DIM, bool FAST>
static bool eta_march_dispatch(int neta, const StepParams& P, const double* eta, const double* p, double* eta_next,
                               double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    switch (neta) {
#define NICR_ETA_CASE(n) \
    case n: launch_eta_march<DIM, FAST, n>(P, eta, p, eta_next, gb_next, s2_next, st, stream); return true;
        NICR_ETA_CASE(1) NICR_ETA_CASE(2) NICR_ETA_CASE(3) NICR_ETA_CASE(4) NICR_ETA_CASE(5) NICR_ETA_CASE(6)
        NICR_ETA_CASE(7) NICR_ETA_CASE(8) NICR_ETA_CASE(9) NICR_ETA_CASE(10) NICR_ETA_CASE(11) NICR_ETA_CASE(12)
        NICR_ETA_CASE(13) NICR_ETA_CASE(14) NICR_ETA_CASE(15) NICR_ETA_CASE(16)
#undef NICR_ETA_CASE
        default: return false;
    }
}

// TMA-staged form of the eta update (3D, row count a multiple of 8, column
// count a multiple of 32, N <= 16 fields), selected by NICR_ETA_KERNEL=tma.
// Measured at 256^3 with 8 fields it is slower than the register march
// (0.72 vs 0.58 ms reciprocal, 1.31 vs 1.15 ms drop-in): the per-plane
// barrier and the seven shared-memory reads per field leave 16 warps per SM
// latency-bound, where the march runs barrier-free from registers and L1. Each CTA owns an 8 x 32 tile and
// marches along its X chunk; one thread stages every plane of all N fields
// with five tensor copies (cp.async.bulk.tensor, the fields as the fourth
// dimension): the tile, the two halo rows (periodic wrap by coordinate) and
// the two 2-column halo strips, into a four-plane shared-memory ring whose
// slots complete on mbarriers. The copy of plane x+2 is issued while plane x
// is updated, and the threads read the stencil from shared memory, so the
// loads hold no registers and cost one instruction per box. Every x
// coordinate is b0, b0 +- 2, b0 + 32, nb - 2 or 0: a multiple of 2 doubles
// (16 bytes) because nb is a multiple of 32. Waits are bounded: a wait that
// runs out sets st->timeout, and the CTA returns after a bounded wait for its
// copies in flight. The arithmetic is the other forms' (same operand order).
__device__ __forceinline__ unsigned smem_u32(const void* ptr) { return (unsigned)__cvta_generic_to_shared(ptr); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

constexpr int kTmaRing = 4;
constexpr long long kTmaWaitLimit = 1LL << 22;   // try_wait rounds before a wait is declared lost

template <int N>
struct TmaStage {
    static constexpr int TA = 8, TB = 32;
    static constexpr int INT = N * TA * TB, ROW = N * TB, COL = N * TA * 2;
    static constexpr int DOUBLES = INT + 2 * ROW + 2 * COL;   // 128-byte multiple for every N
    static constexpr unsigned BYTES = DOUBLES * 8;
    static constexpr size_t SMEM = (size_t)kTmaRing * BYTES + 128;   // + alignment slack
};

template <bool FAST, int N>
__global__ void __launch_bounds__(256, 2)
k_eta_tma(const StepParams P, const __grid_constant__ CUtensorMap m_int, const __grid_constant__ CUtensorMap m_row,
          const __grid_constant__ CUtensorMap m_col, const double* __restrict__ p, double* __restrict__ eta_next,
          double* __restrict__ gb_next, double* __restrict__ s2_next, Status* st) {
    using S = TmaStage<N>;
    constexpr int TA = S::TA, TB = S::TB;
    extern __shared__ unsigned char tma_smem_raw[];
    __shared__ unsigned long long bars[kTmaRing];
    if (st->failed) return;
    const Grid& g = P.g;
    double* ring = reinterpret_cast<double*>(((unsigned long long)tma_smem_raw + 127ull) & ~127ull);
    const int ta = threadIdx.y, tb = threadIdx.x, tid = tb + TB * ta;
    const int a0 = blockIdx.y * TA, b0 = blockIdx.x * TB;
    const int i0 = blockIdx.z * P.xchunk, i1 = min(g.nx, i0 + P.xchunk);
    const int row = a0 + ta, col = b0 + tb;
    const int ytop = a0 == 0 ? g.na - 1 : a0 - 1, ybot = a0 + TA == g.na ? 0 : a0 + TA;
    const int xl = b0 == 0 ? g.nb - 2 : b0 - 2, xr = b0 + TB == g.nb ? 0 : b0 + TB;
    // plane q >= i0 - 1 lives in ring slot (q - i0 + 1) % kTmaRing
    auto slot_of = [&](int q) { return (q - i0 + 1) % kTmaRing; };
    auto stage_of = [&](int q) { return ring + (size_t)slot_of(q) * S::DOUBLES; };
    auto issue = [&](int q) {   // thread 0
        const int xg = q < 0 ? 0 : (q > g.nx - 1 ? g.nx - 1 : q);
        double* s = stage_of(q);
        unsigned long long* bar = &bars[slot_of(q)];
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, S::BYTES);
        tma_load_4d(s, &m_int, b0, a0, xg, 0, bar);
        tma_load_4d(s + S::INT, &m_row, b0, ytop, xg, 0, bar);
        tma_load_4d(s + S::INT + S::ROW, &m_row, b0, ybot, xg, 0, bar);
        tma_load_4d(s + S::INT + 2 * S::ROW, &m_col, xl, a0, xg, 0, bar);
        tma_load_4d(s + S::INT + 2 * S::ROW + S::COL, &m_col, xr, a0, xg, 0, bar);
    };
    bool ok = true;
    auto wait = [&](int q) {
        const int k = q - i0 + 1;
        const unsigned parity = (unsigned)((k / kTmaRing) & 1);
        unsigned long long* bar = &bars[k % kTmaRing];
        for (long long it = 0; ok && !mbar_try_wait(bar, parity); ++it)
            if (it > kTmaWaitLimit) ok = false;
    };
    if (tid == 0) {
        for (int r = 0; r < kTmaRing; ++r) mbar_init(&bars[r], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    int issued = i0 - 2;   // last plane whose copy was issued
    if (tid == 0) {
        for (int q = i0 - 1; q <= i0 + 1 && q <= i1; ++q) issue(q);
    }
    issued = min(i0 + 1, i1);
    wait(i0 - 1);
    wait(i0);
    const long long own = (long long)row * g.pb + col;
    const int c = ta * TB + tb;   // own point in the tile
    unsigned long long errkey = ERR_NONE;
    int x = i0;
    for (; x < i1; ++x) {
        // all threads finished plane x-1 (the slot of plane x+2 held plane x-2)
        if (__syncthreads_or(!ok)) break;
        if (x + 2 <= i1) {
            if (tid == 0) issue(x + 2);
            issued = x + 2;
        }
        wait(x + 1);
        if (!ok) continue;   // reported at the next barrier
        const double* sm = stage_of(x - 1);
        const double* s0 = stage_of(x);
        const double* sp = stage_of(x + 1);
        const double* top = s0 + S::INT;
        const double* bot = top + S::ROW;
        const double* lft = bot + S::ROW;
        const double* rgt = lft + S::COL;
        const long long base = (long long)x * g.plane;
        const double phi = __ldg(p + base + own);
        double S2 = 0.;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const double v = s0[q * TA * TB + c];
            S2 += v * v;
        }
        const long long cell = ((long long)x * g.na + row) * g.nb + col;
        double Sn = 0., pairs = 0.;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const int o = q * TA * TB;
            const double c0 = s0[o + c];
            const double am = ta == 0 ? top[q * TB + tb] : s0[o + c - TB];
            const double ap = ta == TA - 1 ? bot[q * TB + tb] : s0[o + c + TB];
            const double bm = tb == 0 ? lft[(q * TA + ta) * 2 + 1] : s0[o + c - 1];
            const double bp = tb == TB - 1 ? rgt[(q * TA + ta) * 2] : s0[o + c + 1];
            const double lap = fdiv<FAST>((sp[o + c] - 2. * c0 + sm[o + c]), P.v_dxdx)
                             + fdiv<FAST>((ap - 2. * c0 + am), P.v_dada)
                             + fdiv<FAST>((bp - 2. * c0 + bm), P.v_dbdb);
            const double force = grain_deta(c0, S2, phi, P.eta_W, P.eta_A) - P.eta_K * lap;
            const double v = c0 - P.dt_etaL * force;
            if (!isfinite(v) || v < -1.e-12 || v > 1. + 1.e-12)
                errkey = min(errkey, ERR_ETA_BASE + (unsigned long long)q * (unsigned long long)g.ncells + (unsigned long long)cell);
            eta_next[(long long)q * g.nstore + base + own] = v;
            const double sq = v * v;
            pairs += Sn * sq;
            Sn += sq;
        }
        s2_next[base + own] = Sn;
        gb_next[base + own] = P.eta_scale * smin(1., 16. * pairs);
    }
    if (__syncthreads_or(!ok)) {
        // a wait ran out: flag it, give the copies in flight a bounded time to land, leave
        if (tid == 0) {
            atomicOr(&st->timeout, 1);
            for (int q = i0 - 1; q <= issued; ++q) {
                const int k = q - i0 + 1;
                unsigned long long* bar = &bars[k % kTmaRing];
                for (long long it = 0; it <= kTmaWaitLimit && !mbar_try_wait(bar, (unsigned)((k / kTmaRing) & 1)); ++it) {
                }
            }
        }
        __syncthreads();
        return;
    }
    if (errkey != ERR_NONE) atomicMin(&st->err_key, errkey);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the CUDA runtime statically and not libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// The N eta fields of one buffer as a 4D tensor (columns, rows, planes,
// fields), boxes of bx x by x 1 x bw (bw = N: every field at once).
static bool encode_eta_map(CUtensorMap* m, const Grid& g, int n, const double* eta, unsigned bx, unsigned by,
                           unsigned bw) {
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nb, (cuuint64_t)g.na, (cuuint64_t)g.nx, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)g.pb * 8, (cuuint64_t)g.plane * 8, (cuuint64_t)g.nstore * 8};
    const cuuint32_t box[4] = {bx, by, 1, bw};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(eta), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launches the TMA-staged eta update when the grid allows it; false otherwise.
template <bool FAST, int N>
static bool launch_eta_tma_n(const StepParams& P, const double* eta, const double* p, double* eta_next,
                             double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    const Grid& g = P.g;
    CUtensorMap mi, mr, mc;
    if (!encode_eta_map(&mi, g, N, eta, 32, 8, N) || !encode_eta_map(&mr, g, N, eta, 32, 1, N) ||
        !encode_eta_map(&mc, g, N, eta, 2, 8, N))
        return false;
    const size_t smem = TmaStage<N>::SMEM;
    ensure_smem_attr((const void*)k_eta_tma<FAST, N>, (int)smem);
    const dim3 grid(g.nb / 32, g.na / 8, (g.nx + P.xchunk - 1) / P.xchunk);
    k_eta_tma<FAST, N><<<grid, dim3(32, 8), smem, stream>>>(P, mi, mr, mc, p, eta_next, gb_next, s2_next, st);
    return true;
}

template <bool FAST>
static bool launch_eta_tma(int neta, const StepParams& P, const double* eta, const double* p, double* eta_next,
                           double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    const Grid& g = P.g;
    if (g.dim != 3 || g.nb % 32 != 0 || g.na % 8 != 0 || g.nb < 32 || neta < 1 || neta > 16) return false;
    if ((reinterpret_cast<unsigned long long>(eta) & 15ull) != 0) return false;
    switch (neta) {
#define NICR_TMA_CASE(n) \
    case n: return launch_eta_tma_n<FAST, n>(P, eta, p, eta_next, gb_next, s2_next, st, stream);
        NICR_TMA_CASE(1) NICR_TMA_CASE(2) NICR_TMA_CASE(3) NICR_TMA_CASE(4) NICR_TMA_CASE(5) NICR_TMA_CASE(6)
        NICR_TMA_CASE(7) NICR_TMA_CASE(8) NICR_TMA_CASE(9) NICR_TMA_CASE(10) NICR_TMA_CASE(11) NICR_TMA_CASE(12)
        NICR_TMA_CASE(13) NICR_TMA_CASE(14) NICR_TMA_CASE(15) NICR_TMA_CASE(16)
#undef NICR_TMA_CASE
        default: return false;
    }
}

// Streaming form of the eta update: each CTA owns a rows x columns tile,
// marches along X and stages every eta plane once (radius-1 halo) in a
// three-plane shared-memory ring, so every field is read from HBM about once.
// S = sum eta_g^2 is rebuilt from the staged centres in g order, which is the
// same arithmetic as rebuild_eta_mask and therefore the same value as eta_s2.
template <int DIM, int TA, int TB, bool FAST>
__global__ void __launch_bounds__(TA * TB)
k_eta_stream(const StepParams P, int neta, const double* __restrict__ eta, const double* __restrict__ p,
             double* __restrict__ eta_next, double* __restrict__ gb_next, double* __restrict__ s2_next,
             Status* st) {
    constexpr int HA = DIM == 3 ? 1 : 0;
    constexpr int RA = TA + 2 * HA, RB = TB + 2, S1 = RA * RB, NT = TA * TB;
    extern __shared__ __align__(16) double ring[];   // [3][neta][S1], then S1 int offsets
    if (st->failed) return;
    const Grid& g = P.g;
    const int ta = DIM == 3 ? threadIdx.y : 0, tb = threadIdx.x;
    const int a0 = DIM == 3 ? blockIdx.y * TA : 0, b0 = blockIdx.x * TB;
    const int i0 = blockIdx.z * P.xchunk, i1 = min(g.nx, i0 + P.xchunk);
    const int row = a0 + ta, col = b0 + tb;
    const bool active = (DIM == 3 ? row < g.na : true) && col < g.nb;
    const int tid = threadIdx.x + TB * threadIdx.y;
    int* toff = reinterpret_cast<int*>(ring + (size_t)3 * neta * S1);
    for (int r = tid; r < S1; r += NT) {
        const int a = r / RB - HA, b = r % RB - 1;
        toff[r] = (DIM == 3 ? wrapi(a0 + a, g.na) : 0) * g.pb + wrapi(b0 + b, g.nb);
    }
    __syncthreads();
    auto slot = [&](int x) { return ring + (size_t)(((x % 3) + 3) % 3) * neta * S1; };
    auto load = [&](int x) {
        const int xg = x < 0 ? 0 : (x > g.nx - 1 ? g.nx - 1 : x);
        double* dst = slot(x);
        const double* src = eta + (long long)xg * g.plane;
        for (int e = 0; e < neta; ++e) {
            const double* se = src + (long long)e * g.nstore;
            double* de = dst + e * S1;
            for (int r = tid; r < S1; r += NT) de[r] = __ldg(se + toff[r]);
        }
    };
    const int c1 = (ta + HA) * RB + (tb + 1);
    const int bp = c1 + 1, bm = c1 - 1, ap = c1 + RB, am = c1 - RB;
    unsigned long long errkey = ERR_NONE;
    load(i0 - 1);
    load(i0);
    for (int u = i0; u < i1; ++u) {
        load(u + 1);
        __syncthreads();
        if (active) {
            const double* sm = slot(u - 1);
            const double* s0 = slot(u);
            const double* sp = slot(u + 1);
            const long long idx = (long long)u * g.plane + (long long)row * g.pb + col;
            const long long cell = ((long long)u * g.na + row) * g.nb + col;
            double S = 0.;
            for (int e = 0; e < neta; ++e) {
                const double v = s0[e * S1 + c1];
                S += v * v;
            }
            const double phi = __ldg(p + idx);
            double Sn = 0., pairs = 0.;
            for (int e = 0; e < neta; ++e) {
                const int o = e * S1;
                const double ec = s0[o + c1];
                double lap;
                if (DIM == 3)
                    lap = fdiv<FAST>((sp[o + c1] - 2. * ec + sm[o + c1]), P.v_dxdx)
                        + fdiv<FAST>((s0[o + ap] - 2. * ec + s0[o + am]), P.v_dada)
                        + fdiv<FAST>((s0[o + bp] - 2. * ec + s0[o + bm]), P.v_dbdb);
                else
                    lap = fdiv<FAST>((sp[o + c1] - 2. * ec + sm[o + c1]), P.v_dxdx)
                        + fdiv<FAST>((s0[o + bp] - 2. * ec + s0[o + bm]), P.v_dbdb);
                const double force = grain_deta(ec, S, phi, P.eta_W, P.eta_A) - P.eta_K * lap;
                const double v = ec - P.dt_etaL * force;
                if (!isfinite(v) || v < -1.e-12 || v > 1. + 1.e-12)
                    errkey = min(errkey, ERR_ETA_BASE + (unsigned long long)e * (unsigned long long)g.ncells + (unsigned long long)cell);
                eta_next[(long long)e * g.nstore + idx] = v;
                const double sq = v * v;
                pairs += Sn * sq;
                Sn += sq;
            }
            s2_next[idx] = Sn;
            gb_next[idx] = P.eta_scale * smin(1., 16. * pairs);
        }
        __syncthreads();   // slot(u-1) is refilled with plane u+2 next
    }
    if (errkey != ERR_NONE) atomicMin(&st->err_key, errkey);
}

// Batched step: one launch advances up to kBatchMax domains of one
// dimensionality and arithmetic form. The per-domain parameters and buffers
// sit in the kernel's parameter space (read through the constant cache with a
// block-uniform index); block b belongs to the last domain whose first block
// is <= b and runs exactly the CTA (bx, by, bz) the single-domain launch would
// run, with the same partial-sum slot, so every domain's result is identical
// to its own nicr_step.
// The compact batch: the block's domain's parameters are the shared ones with
// the domain's grid, inlet value and ranges.
template <int DIM, int TA, int TB, int MINB, bool FAST>
__global__ void __launch_bounds__(TA * TB, MINB) k_step_batch_slim(const __grid_constant__ StepBatchSlim B) {
    int lo = 0, hi = B.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (B.d[mid].block0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BatchSlim& D = B.d[lo];
    StepParams P = B.base;
    P.g = D.g;
    P.layer_o = D.layer_o;
    P.inlet = D.inlet;
    P.x_hi = D.x_hi;
    P.key_ncells = D.key_ncells;
    const int t = (int)blockIdx.x - D.block0;
    const int bx = t % D.gx, r = t / D.gx, by = r % D.gy, bz = r / D.gy;
    StepKernel<DIM, TA, TB, FAST>::run(P, D.o, D.cr, D.p, D.gb, D.s2, D.on, D.crn, D.pn, D.partials, D.st, bx, by,
                                       bz, t);
}

template <int DIM, int TA, int TB, int MINB, bool FAST>
__global__ void __launch_bounds__(TA * TB, MINB) k_step_batch(const __grid_constant__ StepBatch B) {
    int lo = 0, hi = B.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (B.d[mid].block0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BatchDomain& D = B.d[lo];
    const int t = (int)blockIdx.x - D.block0;
    const int bx = t % D.gx, r = t / D.gx, by = r % D.gy, bz = r / D.gy;
    StepKernel<DIM, TA, TB, FAST>::run(D.sp, D.o, D.cr, D.p, D.gb, D.s2, D.on, D.crn, D.pn, D.partials, D.st, bx, by,
                                       bz, t);
}

}  // namespace

// X chunk of the step and eta kernels. A CTA marching c planes also computes
// mu and M of the plane before its chunk and stages that plane's halo, about
// two planes of extra work, and CTAs run in waves of 2 (3D) or 4 (2D) per SM,
// so the chunk minimising waves x (c + 2) is taken among nx halved repeatedly
// and the powers of two below nx, the longer chunk on ties. Small domains get short chunks and use the whole GPU
// (2D 128^2: 1 plane per CTA; 64^3: 4), large ones long chunks (256^3: 32).
// NICR_XCHUNK forces a chunk for tuning runs.
// Occupancy variant of the 3D step kernel: 2 CTAs/SM (no register cap, the
// default: with the staging loads software-pipelined it is measured faster on
// B200) or 3 CTAs/SM (80 registers, which spills). NICR_STEP_MINB=2|3 selects
// one for tuning runs.
static int step_minb() {
    static int v = 0;
    if (!v) {
        const char* e = getenv("NICR_STEP_MINB");
        v = (e && e[0] == '3') ? 3 : 2;
    }
    return v;
}
static int step_minb_for(const StepParams& P) { return P.minb == 2 || P.minb == 3 ? P.minb : step_minb(); }

// CTAs per SM of the recomputation kernel (its grid strides over the step grid)
constexpr int kRedoCtasPerSm = 2;

template <int MINB, bool FAST>
static void launch_step3(const StepParams& P, const double* o, const double* cr, const double* p, const double* gb,
                         const double* s2, double* on, double* crn, double* pn, StepPartial* partials, Status* st,
                         cudaStream_t stream, int* nblocks_out) {
    using T = Tile<3, TA3, TB3>;
    const dim3 grid = step_grid<3, TA3, TB3>(P);
    const int nblocks = (int)(grid.x * grid.y * grid.z);
    const int gredo = std::min(nblocks, kRedoCtasPerSm * 148);
    if (P.err_slot >= 0) {   // an X slab
        ensure_smem_attr((const void*)k_step_main<3, TA3, TB3, MINB, FAST, true>, (int)T::SMEM_BYTES);
        k_step_main<3, TA3, TB3, MINB, FAST, true><<<grid, dim3(TB3, TA3), T::SMEM_BYTES, stream>>>(
            P, o, cr, p, gb, s2, on, crn, pn, partials, st);
        if constexpr (!FAST) {
            ensure_smem_attr((const void*)k_step_redo<3, TA3, TB3, true>, (int)T::SMEM_BYTES);
            k_step_redo<3, TA3, TB3, true><<<gredo, dim3(TB3, TA3), T::SMEM_BYTES, stream>>>(
                P, o, cr, p, gb, s2, on, crn, pn, partials, st, (int)grid.x, (int)grid.y, nblocks);
        }
    } else {
        ensure_smem_attr((const void*)k_step_main<3, TA3, TB3, MINB, FAST>, (int)T::SMEM_BYTES);
        k_step_main<3, TA3, TB3, MINB, FAST><<<grid, dim3(TB3, TA3), T::SMEM_BYTES, stream>>>(P, o, cr, p, gb, s2, on,
                                                                                             crn, pn, partials, st);
        if constexpr (!FAST) {
            ensure_smem_attr((const void*)k_step_redo<3, TA3, TB3>, (int)T::SMEM_BYTES);
            k_step_redo<3, TA3, TB3><<<gredo, dim3(TB3, TA3), T::SMEM_BYTES, stream>>>(
                P, o, cr, p, gb, s2, on, crn, pn, partials, st, (int)grid.x, (int)grid.y, nblocks);
        }
    }
    if (nblocks_out) *nblocks_out = nblocks;
}

template <bool FAST>
static void launch_step_form(const StepParams& P, const double* o, const double* cr, const double* p,
                             const double* gb, const double* s2, double* on, double* crn, double* pn,
                             StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out) {
    if (P.g.dim == 3) {
        if (step_minb_for(P) == 3) launch_step3<3, FAST>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, stream, nblocks_out);
        else launch_step3<2, FAST>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, stream, nblocks_out);
    } else {
        using T = Tile<2, TA2, TB2>;
        const dim3 grid = step_grid<2, TA2, TB2>(P);
        k_step_main<2, TA2, TB2, 4, FAST><<<grid, dim3(TB2, TA2), T::SMEM_BYTES, stream>>>(P, o, cr, p, gb, s2, on,
                                                                                          crn, pn, partials, st);
        const int nblocks = (int)(grid.x * grid.y * grid.z);
        if constexpr (!FAST)
            k_step_redo<2, TA2, TB2><<<std::min(nblocks, kRedoCtasPerSm * 148), dim3(TB2, TA2), T::SMEM_BYTES,
                                       stream>>>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, (int)grid.x,
                                                 (int)grid.y, nblocks);
        if (nblocks_out) *nblocks_out = nblocks;
    }
}

template <bool FAST>
static void launch_eta_form(const StepParams& P, int neta, const double* eta, const double* s2, const double* p,
                            double* eta_next, double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    const Grid& g = P.g;
    // The streaming kernel stalls on its per-plane barriers until the next
    // plane has arrived; it is kept only as a tuning option.
    // Kernel choice (measured on B200 at 256^3 with 8 fields): the X-marching
    // kernel for the reciprocal form (0.63 ms vs 0.94 ms per step), the
    // per-cell kernel for the drop-in form, where the unrolled verified
    // divisions of the marching kernel cost more than its saved loads (1.84 ms
    // vs 1.29 ms). NICR_ETA_KERNEL=march|simple|stream overrides for tuning.
    static int simple = -1, march = -1, tma = -1;
    if (simple < 0) {
        const char* e = getenv("NICR_ETA_KERNEL");
        simple = (e && e[0] == 's' && e[1] == 't') ? 0 : 1;
        march = e ? (e[0] == 'm' ? 1 : 0) : -2;
        tma = (e && e[0] == 't') ? 1 : 0;
    }
    const bool slab = P.err_slot >= 0;   // X slabs use the march or the per-cell kernel
    if (tma && !slab && launch_eta_tma<FAST>(neta, P, eta, p, eta_next, gb_next, s2_next, st, stream)) return;
    if (march == 1 || (march == -2 && FAST)) {
        const bool done = g.dim == 3 ? eta_march_dispatch<3, FAST>(neta, P, eta, p, eta_next, gb_next, s2_next, st, stream)
                                     : eta_march_dispatch<2, FAST>(neta, P, eta, p, eta_next, gb_next, s2_next, st, stream);
        if (done) return;
    }
    if (g.dim == 3) {
        constexpr int TA = 8, TB = 32, S1 = (TA + 2) * (TB + 2);
        const size_t smem = (size_t)3 * neta * S1 * sizeof(double) + S1 * sizeof(int);
        if (!simple && !slab && smem <= 200 * 1024) {
            ensure_smem_attr((const void*)k_eta_stream<3, TA, TB, FAST>, 200 * 1024);
            const dim3 grid((g.nb + TB - 1) / TB, (g.na + TA - 1) / TA, (g.nx + P.xchunk - 1) / P.xchunk);
            k_eta_stream<3, TA, TB, FAST><<<grid, dim3(TB, TA), smem, stream>>>(P, neta, eta, p, eta_next, gb_next, s2_next, st);
            return;
        }
        const dim3 block(32, 8);
        const dim3 grid((g.nb + 31) / 32, (g.na + 7) / 8, P.x_hi - P.x_lo);
        k_eta_update<3, FAST><<<grid, block, 0, stream>>>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, st);
    } else {
        constexpr int TB = 128, S1 = TB + 2;
        const size_t smem = (size_t)3 * neta * S1 * sizeof(double) + S1 * sizeof(int);
        if (!simple && smem <= 200 * 1024) {
            ensure_smem_attr((const void*)k_eta_stream<2, 1, TB, FAST>, 200 * 1024);
            const dim3 grid((g.nb + TB - 1) / TB, 1, (g.nx + P.xchunk - 1) / P.xchunk);
            k_eta_stream<2, 1, TB, FAST><<<grid, dim3(TB, 1), smem, stream>>>(P, neta, eta, p, eta_next, gb_next, s2_next, st);
            return;
        }
        const dim3 block(128, 1);
        const dim3 grid((g.nb + 127) / 128, 1, g.nx);
        k_eta_update<2, FAST><<<grid, block, 0, stream>>>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, st);
    }
}

template <int DIM, int TA, int TB, int MINB, bool FAST>
static void launch_batch_slim(const StepBatchSlim& B, int nblocks, cudaStream_t stream) {
    using T = Tile<DIM, TA, TB>;
    ensure_smem_attr((const void*)k_step_batch_slim<DIM, TA, TB, MINB, FAST>, (int)T::SMEM_BYTES);
    k_step_batch_slim<DIM, TA, TB, MINB, FAST><<<nblocks, dim3(TB, TA), T::SMEM_BYTES, stream>>>(B);
}

template <int DIM, int TA, int TB, int MINB, bool FAST>
static void launch_batch_group(StepBatch& B, int nblocks, cudaStream_t stream) {
    using T = Tile<DIM, TA, TB>;
    ensure_smem_attr((const void*)k_step_batch<DIM, TA, TB, MINB, FAST>, (int)T::SMEM_BYTES);
    k_step_batch<DIM, TA, TB, MINB, FAST><<<nblocks, dim3(TB, TA), T::SMEM_BYTES, stream>>>(B);
}

}  // namespace nicr
