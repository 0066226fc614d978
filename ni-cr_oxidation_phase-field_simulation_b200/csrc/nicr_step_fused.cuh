// One HBM pass per step in 3D with evolving eta: the step kernel and the eta
// update fused into one X march (the reference's refresh + step + eta_trial,
// 3S:597-620, 3S:761-826, 3S:514-526, with rebuild_eta_mask 3S:495-507 done
// on chip). Included by nicr_step_impl.cuh users after the shared templates.
//
// Per CTA: a 16 x 32 tile (512 threads, one CTA per SM) marching along its X
// chunk. o, cr and phi are staged as in k_step_main (register prefetch into
// shared-memory rings). The N eta fields of each plane are staged by TMA
// (cp.async.bulk.tensor, five boxes per field: the tile, the two wrapped halo
// rows and the two 2-column halo strips, issued by one lane per field, and
// four corner boxes of all fields) into a three-plane ring whose slots
// complete on mbarriers. Each field's tile and halo form one block at a fixed
// stride, so every stencil read is a shared load at a per-thread base plus a
// compile-time offset. The copy of plane u+2 is
// issued at the top of the iteration that updates plane u, one plane ahead of
// its use. From the staged plane of the lead plane x every thread
// rebuilds S = sum eta^2 and the GB mask gb = scale*min(1,16*pairs) at its own
// point and, for the first 100 threads, at one halo-ring point, in
// rebuild_eta_mask's order, so the mobilities of the lead plane need no gb
// array and the phi force no eta_s2 array. The eta update of plane u reads
// its centre and in-plane neighbours from the slot of plane u, the +X value
// from the slot of plane u+1 and the -X value from registers (each thread's
// own column of plane u-1, kept from the previous iteration).
//
// HBM traffic per cell and step: o, cr, phi and the N eta read once and
// written once: (6 + 2N) * 8 bytes (176 at N = 8), against (6 + 2N) * 8 + 40
// for the two-kernel form, which writes and re-reads gb and eta_s2 and reads
// phi twice. The handle's gb and eta_s2 arrays are not written; the model
// rebuilds them (k_eta_mask) when something reads them.
//
// Shared memory at N = 8: 102.8 KB of step staging + 3 x 42 KB of eta slots
// = 226 KB, so N <= 8 and one CTA per SM. Grids: rows a multiple of 16,
// columns a multiple of 32 (whole tiles, so every TMA box and its x
// coordinate, b0, b0 - 2, b0 + 32, nb - 2 or 0, is a multiple of two doubles).
// Every mbarrier wait is bounded; a wait that runs out sets st->timeout and
// the CTA leaves after a bounded wait for its own copies in flight.
#pragma once

namespace nicr {
namespace {

// A field stride known at compile time (the own point's), converting like an int.
template <int S>
struct ConstStride {
    __device__ __forceinline__ operator int() const { return S; }
};

constexpr int FTA = 16, FTB = 32;    // fused tile: 16 rows x 32 columns
constexpr int kFusedMaxEta = 8;

template <int N>
struct FusedLayout {
    static constexpr int TA = FTA, TB = FTB, NT = TA * TB;
    // One field's block in an eta slot (doubles; every TMA region starts on a
    // 128-byte boundary): tile [TA][TB], top and bottom halo rows [TB], left
    // and right strips [TA][2] (columns b0-2, b0-1 and b0+32, b0+33); FS
    // doubles per field. After the N blocks, the corners (-1,-1), (-1,TB),
    // (TA,-1), (TA,TB) of all fields, one [N][2] box each (columns as the
    // strips), CP doubles apart.
    static constexpr int O_TOP = NT, O_BOT = O_TOP + TB, O_LFT = O_BOT + TB, O_RGT = O_LFT + 2 * TA;
    static constexpr int FS = O_RGT + 2 * TA;
    static constexpr int CP = (2 * N + 15) / 16 * 16;
    static constexpr int O_CRN = N * FS;
    static constexpr int SLOT = O_CRN + 4 * CP;
    static constexpr unsigned TX_BYTES = (unsigned)N * (NT + 2 * TB + 4 * TA + 8) * 8u;   // the TMA boxes of a slot
    static constexpr int RING = 3;
    using T = Tile<3, TA, TB>;
    // step staging (T::SMEM_DOUBLES) + the block reduction's scratch (32 warps x 5 DD + counts)
    static constexpr size_t STEP_BYTES = ((size_t)T::SMEM_DOUBLES * 8 + 32 * (5 * 16 + 8) + 127) / 128 * 128;
    static constexpr size_t BYTES = STEP_BYTES + 128 + (size_t)RING * SLOT * 8;
    static_assert(O_TOP % 16 == 0 && O_BOT % 16 == 0 && O_LFT % 16 == 0 && O_RGT % 16 == 0 && FS % 16 == 0 &&
                  CP % 16 == 0, "TMA destinations must stay 128-byte aligned");
};

// Offset of a point of the tile + halo ring in an eta slot, field 0; field q
// lies stride * q further (FS, or 2 for the corners).
template <int N>
__device__ __forceinline__ int eta_slot_point(int a, int b, int& stride) {
    using L = FusedLayout<N>;
    constexpr int TA = L::TA, TB = L::TB;
    stride = L::FS;
    if (a >= 0 && a < TA && b >= 0 && b < TB) return a * TB + b;
    if (b >= 0 && b < TB) return (a < 0 ? L::O_TOP : L::O_BOT) + b;
    if (a >= 0 && a < TA) return b < 0 ? L::O_LFT + a * 2 + 1 : L::O_RGT + a * 2;
    stride = 2;
    return L::O_CRN + ((a < 0 ? 0 : 2) + (b < 0 ? 0 : 1)) * L::CP + (b < 0 ? 1 : 0);
}

// MODE 1: O diffusion on, legacy Ck, legacy bounds (the common setting, the
// benchmark's): those flags fold at compile time; MODE 0 reads them from P.
template <bool FAST, int N, int MODE>
struct OnePassStep {
    using L = FusedLayout<N>;
    using T = typename L::T;
    using SK = StepKernel<3, FTA, FTB, FAST>;
    static constexpr int TA = FTA, TB = FTB, NT = L::NT;

    // S and the GB mask of one point from a staged eta plane (rebuild_eta_mask order)
    template <typename Stride>
    __device__ static double mask_at(const StepParams& P, const double* slot, int off, Stride stride, double& S) {
        double s = 0., pairs = 0.;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const double e = slot[off + q * stride];
            const double sq = e * e;
            pairs += s * sq;
            s += sq;
        }
        S = s;
        return P.eta_scale * smin(1., 16. * pairs);
    }

    // o, cr at plane xoc (radius 2) and phi at plane xp (radius 1) into registers
    __device__ static void fetch_ocp(const StepParams& P, const double* __restrict__ o, const double* __restrict__ cr,
                                     const double* __restrict__ p, int xoc, int xp, const typename SK::Offs& f,
                                     typename SK::Prefetch& r) {
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

    // One march over the CTA's chunk with the division policy of DM (DivOf).
    // kb offsets the staging ring's plane counter (slot and phase of each
    // copy), so a second march continues the mbarrier phases of the first;
    // DM 1 returns true, without publishing keys or partials, when a
    // numerator of the chunk left the exact-division range.
    template <int DM>
    __device__ static bool run_body(const StepParams& P, const CUtensorMap* m_int, const CUtensorMap* m_row,
                                    const CUtensorMap* m_col, const CUtensorMap* m_crn, const double* __restrict__ o,
                                    const double* __restrict__ cr, const double* __restrict__ p,
                                    double* __restrict__ on, double* __restrict__ crn, double* __restrict__ pn,
                                    double* __restrict__ eta_next, StepPartial* __restrict__ partials, Status* st,
                                    unsigned long long* bars, int kb) {
        extern __shared__ __align__(128) unsigned char fused_smem[];
        double* smem = reinterpret_cast<double*>(fused_smem);
        double* so = smem;                 // 4 slots x S2
        double* scr = so + 4 * T::S2;      // 4 slots x S2
        double* sp = scr + 4 * T::S2;      // 3 slots x S1
        double* smuO = sp + 3 * T::S1;     // 2 slots x S1
        double* smuCr = smuO + 2 * T::S1;
        double* smo = smuCr + 2 * T::S1;
        double* smc = smo + 2 * T::S1;
        DD* sdd = reinterpret_cast<DD*>(smc + 2 * T::S1);
        long long* scnt = reinterpret_cast<long long*>(sdd + 32 * 5);
        // the eta ring on a 128-byte boundary (an offset from the shared array, so
        // the compiler keeps shared-memory addressing)
        double* ering = reinterpret_cast<double*>(
            fused_smem + L::STEP_BYTES + ((128u - (smem_u32(fused_smem + L::STEP_BYTES) & 127u)) & 127u));

        if (st->failed) return false;   // a previous step of this batch was rejected
        unsigned dbad = 0;
        const typename DivOf<DM>::T dv{P, dbad};

        const bool o_on = MODE == 1 ? true : P.o_on != 0;
        const bool ck_legacy = MODE == 1 ? true : P.ck == 0;
        const bool bounds_legacy = MODE == 1 ? true : P.bounds == 1;
        const Grid& g = P.g;
        const int ta = threadIdx.y, tb = threadIdx.x, tid = tb + TB * ta;
        const int a0 = blockIdx.y * TA, b0 = blockIdx.x * TB;
        const int i0 = blockIdx.z * P.xchunk, i1 = min(g.nx, i0 + P.xchunk);
        const int row = a0 + ta, col = b0 + tb;
        const typename SK::Offs offs = SK::make_offs(g, a0, b0);

        // ---- eta staging: plane q (clamped to [0, nx-1], the Neumann ghosts)
        // lives in slot (q - i0 + 1) % 3; planes i0-1 .. i1 are staged once each
        const int ytop = a0 == 0 ? g.na - 1 : a0 - 1, ybot = a0 + TA == g.na ? 0 : a0 + TA;
        const int xl = b0 == 0 ? g.nb - 2 : b0 - 2, xr = b0 + TB == g.nb ? 0 : b0 + TB;
        auto eslot = [&](int q) { return ering + (size_t)((q - i0 + 1 + kb) % L::RING) * L::SLOT; };
        // the last warp: lane 0 registers the slot's bytes on its mbarrier, then
        // lane q < N copies field q's five boxes and lanes N .. N+3 the corners
        auto issue = [&](int q) {
            const int lane = tid - (NT - 32);
            if (lane < 0) return;
            const int xg = q < 0 ? 0 : (q > g.nx - 1 ? g.nx - 1 : q);
            double* s = eslot(q);
            unsigned long long* bar = &bars[(q - i0 + 1 + kb) % L::RING];
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_expect_tx(bar, L::TX_BYTES);
            }
            __syncwarp();
            if (lane < N) {
                double* f = s + lane * L::FS;
                tma_load_4d(f, m_int, b0, a0, xg, lane, bar);
                tma_load_4d(f + L::O_TOP, m_row, b0, ytop, xg, lane, bar);
                tma_load_4d(f + L::O_BOT, m_row, b0, ybot, xg, lane, bar);
                tma_load_4d(f + L::O_LFT, m_col, xl, a0, xg, lane, bar);
                tma_load_4d(f + L::O_RGT, m_col, xr, a0, xg, lane, bar);
            } else if (lane < N + 4) {
                const int k = lane - N;
                tma_load_4d(s + L::O_CRN + k * L::CP, m_crn, (k & 1) ? xr : xl, k < 2 ? ytop : ybot, xg, 0, bar);
            }
        };
        bool ok = true;
        auto wait = [&](int q) {
            const int k = q - i0 + 1 + kb;
            const unsigned parity = (unsigned)((k / L::RING) & 1);
            unsigned long long* bar = &bars[k % L::RING];
            for (long long it = 0; ok && !mbar_try_wait(bar, parity); ++it)
                if (it > kTmaWaitLimit) ok = false;
        };
        if (tid == 0 && kb == 0) {
            for (int r = 0; r < L::RING; ++r) mbar_init(&bars[r], 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncthreads();
        int issued = i0 + 1;   // last plane whose copy was issued
        for (int q = i0 - 1; q <= i0 + 1; ++q) issue(q);

        // per-thread positions in an eta slot: own point and its four in-plane
        // neighbours; the halo-ring point of the first S1 - NT threads
        const int e_own = ta * TB + tb;
        int unused;
        const int am_o = eta_slot_point<N>(ta - 1, tb, unused), ap_o = eta_slot_point<N>(ta + 1, tb, unused);
        const int bm_o = eta_slot_point<N>(ta, tb - 1, unused), bp_o = eta_slot_point<N>(ta, tb + 1, unused);
        int ring_o = 0, ring_s = L::FS;
        if (offs.gl[1] >= 0) {
            int a, b;
            SK::ring_point(tid, a, b);
            ring_o = eta_slot_point<N>(a, b, ring_s);
        }

        DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};  // ckO ckCr clipO clipCr bcO
        long long clipped = 0;
        unsigned long long errkey = ERR_NONE;

        auto slot3 = [](int w) { return ((w % 3) + 3) % 3; };
        auto oslot = [&](int w) { return so + (w & 3) * T::S2; };
        auto cslot = [&](int w) { return scr + (w & 3) * T::S2; };
        auto pslot = [&](int x) { return sp + slot3(x) * T::S1; };

        // the lead plane x over the tile + radius-1 halo; S and gb of the own
        // point are returned for the update of plane x in the next iteration
        auto lead = [&](int x, double& S_own, double& gb_own) -> CenterVals {
            const double* es = eslot(x);
            double gbl[2];
            gbl[0] = mask_at(P, es, e_own, ConstStride<L::FS>(), S_own);
            gb_own = gbl[0];
            const double *som = oslot(x - 1), *so0 = oslot(x), *sop = oslot(x + 1);
            const double *scm = cslot(x - 1), *sc0 = cslot(x), *scp = cslot(x + 1);
            const double* spx = pslot(x);
            double* mO = smuO + (x & 1) * T::S1;
            double* mC = smuCr + (x & 1) * T::S1;
            double* mo_ = smo + (x & 1) * T::S1;
            double* mc_ = smc + (x & 1) * T::S1;
            CenterVals own = SK::lead_core(dv, P, o_on, som, so0, sop, scm, sc0, scp, spx, mO, mC, mo_, mc_, ta, tb,
                                           gbl[0]);
            if (offs.gl[1] >= 0) {
                double Sr;
                gbl[1] = mask_at(P, es, ring_o, ring_s, Sr);
                int a, b;
                SK::ring_point(tid, a, b);
                SK::lead_core(dv, P, o_on, som, so0, sop, scm, sc0, scp, spx, mO, mC, mo_, mc_, a, b, gbl[1]);
            }
            return own;
        };

        double pP, FxO, FxCr;   // phi of plane u-1 (own point), left x-face fluxes of plane u
        double s2u, gbu;          // S and gb of the own point of the update plane
        double ep[N];             // own column of eta at plane u - 1
        // ---- prologue: centre values of the first update plane and its left x-face flux
        if (i0 == 0) {
            SK::load_oc(P, o, cr, -1, oslot(-1), cslot(-1), offs);
            SK::load_oc(P, o, cr, 0, oslot(0), cslot(0), offs);
            SK::load_oc(P, o, cr, 1, oslot(1), cslot(1), offs);
            SK::load_p(P, p, 0, pslot(0), offs);
            wait(-1);
            wait(0);
            __syncthreads();
            const CenterVals C = lead(0, s2u, gbu);
            __syncthreads();
            const double muOg = (P.bc == 1 && o_on) ? 2. * P.mu_res - C.muO : C.muO;
            FxO = dv.dvx(-.5 * (C.mo + C.mo) * (C.muO - muOg));
            FxCr = dv.dvx(-.5 * (C.mc + C.mc) * (C.muCr - C.muCr));
            pP = C.p;
            // the x = 0 face of plane 0 and the inlet's budget term, here rather
            // than in the march: left_flux (3S:621-628), the surface-mobility
            // closure of the O face with bc=mu, replaces the ghost face
            if (P.bc == 1) {
                double lf = 0.;
                if (o_on) {
                    const double mf = mobility(P.surface_c_ref, h(C.p), gbu, Phys::bmo, Phys::boo, P.gbm1_o);
                    lf = dv.dvx(2. * mf * (P.mu_res - C.muO));
                }
                FxO = lf;
                acc[4] = dd_add(acc[4], dv.dvx(P.dt * lf));
            }
            if (P.inlet) acc[4] = dd_add(acc[4], P.layer_o - __ldg(o + (long long)row * g.pb + col));
        } else {
            SK::load_oc(P, o, cr, i0 - 2, oslot(i0 - 2), cslot(i0 - 2), offs);
            SK::load_oc(P, o, cr, i0 - 1, oslot(i0 - 1), cslot(i0 - 1), offs);
            SK::load_oc(P, o, cr, i0, oslot(i0), cslot(i0), offs);
            SK::load_p(P, p, i0 - 1, pslot(i0 - 1), offs);
            wait(i0 - 1);
            __syncthreads();
            double Sm, gbm;
            const CenterVals Pv = lead(i0 - 1, Sm, gbm);
            SK::load_oc(P, o, cr, i0 + 1, oslot(i0 + 1), cslot(i0 + 1), offs);
            SK::load_p(P, p, i0, pslot(i0), offs);
            wait(i0);
            __syncthreads();
            const CenterVals C = lead(i0, s2u, gbu);
            __syncthreads();
            FxO = dv.dvx(-.5 * (Pv.mo + C.mo) * (C.muO - Pv.muO));
            FxCr = dv.dvx(-.5 * (Pv.mc + C.mc) * (C.muCr - Pv.muCr));
            pP = Pv.p;
        }
        {
            const double* es = eslot(i0 - 1);   // plane i0 - 1 (plane 0, the Neumann ghost, when i0 = 0)
#pragma unroll
            for (int q = 0; q < N; ++q) ep[q] = es[e_own + q * L::FS];
        }

        typename SK::Prefetch pf;
        if (i0 + 1 <= g.nx - 1) fetch_ocp(P, o, cr, p, i0 + 2, i0 + 1, offs, pf);
        for (int u = i0; u < i1; ++u) {
            const int x = u + 1;
            double s2n = 0., gbn = 0.;
            if (x <= g.nx - 1) {
                SK::store(pf, oslot(x + 1), cslot(x + 1), pslot(x), offs);
                // one barrier per plane: this plane's staging before lead(x); the
                // previous iteration's reads of the mu/M slot lead(x) overwrites and
                // of the eta slot the copy of plane u+2 overwrites
                if (__syncthreads_or(!ok)) break;
                if (u + 2 <= i1) {
                    issue(u + 2);
                    issued = u + 2;
                }
                if (x + 1 <= g.nx - 1 && u + 1 < i1) fetch_ocp(P, o, cr, p, x + 2, x + 1, offs, pf);
                wait(x);
                lead(x, s2n, gbn);
            } else {
                if (__syncthreads_or(!ok)) break;
                wait(x);   // plane nx: the clamped copy of plane nx-1 (the eta +X ghost)
            }
            {
                const double* mO = smuO + (u & 1) * T::S1;
                const double* mC = smuCr + (u & 1) * T::S1;
                const double* mo_ = smo + (u & 1) * T::S1;
                const double* mc_ = smc + (u & 1) * T::S1;
                const double* spu = pslot(u);
                const int c1 = T::i1(ta, tb);
                const int bp = T::i1(ta, tb + 1), bm = T::i1(ta, tb - 1);
                const int ap = T::i1(ta + 1, tb), am = T::i1(ta - 1, tb);
                const long long gidx = (long long)u * g.plane + (long long)row * g.pb + col;
                // the cell's index in reference loop order, for failing-trial keys only
                auto cell_of = [&]() { return ((long long)u * g.na + row) * g.nb + col; };
                // Centre (plane u) and lead (plane x) values are read back from
                // the staging rings rather than carried in registers across the
                // iteration (the same doubles; fewer live registers). The ghost
                // plane nx is the Neumann copy of plane nx-1, mu and M included.
                CenterVals C, Lv;
                {
                    const int c2 = T::i2(ta, tb);
                    C.o = oslot(u)[c2]; C.cr = cslot(u)[c2]; C.p = spu[c1]; C.hh = h(C.p);
                    C.muO = mO[c1]; C.muCr = mC[c1]; C.mo = mo_[c1]; C.mc = mc_[c1];
                    if (x <= g.nx - 1) {
                        const int lx = (x & 1) * T::S1 + c1;
                        Lv.p = pslot(x)[c1];
                        Lv.muO = smuO[lx]; Lv.muCr = smuCr[lx]; Lv.mo = smo[lx]; Lv.mc = smc[lx];
                    } else {
                        Lv = C;
                    }
                }

                // fluxes, phi force and Ck (3S:761-811); the trial test and the
                // clamps below without data-dependent branches (so the scheduler
                // sees one block); the rare bookkeeping (budget terms of changed
                // cells, failure keys) is one branch after the stores
                const typename SK::CoreOut R = SK::cell_core(dv, P, o_on, ck_legacy, true, C, Lv, pP, FxO, FxCr, s2u,
                                                             mO, mC, mo_, mc_, spu, c1, bp, bm, ap, am);
                const double pp = C.p;
                double onv = R.onv, crv = R.crv, pnv = R.pnv;
                const double dO = R.dO, dCr = R.dCr, rightO = R.rightO, rightCr = R.rightCr;
                const bool nonfinite = !isfinite(onv) || !isfinite(crv) || !isfinite(pnv);
                double clO = 0., clCr = 0.;
                bool outside = false;
                if (bounds_legacy) {
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
                    if (nonfinite || outside)
                        errkey = min(errkey, (unsigned long long)cell_of() * 4ull + (nonfinite ? 0ull : 1ull));
                    // adding +-0 to a normalised double-double leaves it unchanged,
                    // so zero increments are skipped
                    if (dO != 0.) acc[0] = dd_add(acc[0], dO);
                    if (dCr != 0.) acc[1] = dd_add(acc[1], dCr);
                    if (clO != 0.) acc[2] = dd_add(acc[2], clO);
                    if (clCr != 0.) acc[3] = dd_add(acc[3], clCr);
                }

                // eta_trial (3S:514-526) at plane u: v = eta - (dt L_eta)(deta - K lap eta);
                // the fields failing the range test are collected as bits and keyed
                // once (the first field in reference order)
                {
                    const double* es = eslot(u);
                    const double* en = eslot(u + 1);
                    double* edst = eta_next + gidx;
                    unsigned ebad = 0;
#pragma unroll
                    for (int q = 0; q < N; ++q) {
                        const int fq = q * L::FS;
                        const double c0 = es[e_own + fq];
                        const double lap = dv.dvxx((en[e_own + fq] - 2. * c0 + ep[q]))
                                         + dv.dvaa((es[ap_o + fq] - 2. * c0 + es[am_o + fq]))
                                         + dv.dvbb((es[bp_o + fq] - 2. * c0 + es[bm_o + fq]));
                        const double force = grain_deta(c0, s2u, C.p, P.eta_W, P.eta_A) - P.eta_K * lap;
                        const double v = c0 - P.dt_etaL * force;
                        ebad |= (!isfinite(v) || v < -1.e-12 || v > 1. + 1.e-12) ? (1u << q) : 0u;
                        *edst = v;
                        edst += g.nstore;
                        ep[q] = c0;
                    }
                    if (ebad)
                        errkey = min(errkey, ERR_ETA_BASE + (unsigned long long)(__ffs(ebad) - 1) *
                                                 (unsigned long long)g.ncells + (unsigned long long)cell_of());
                }

                pP = pp;   // a register: the ring slot of plane u-1 takes plane u+2 next
            }
            s2u = s2n;
            gbu = gbn;
        }
        if (__syncthreads_or(!ok)) {
            // a wait ran out: flag it, give the copies in flight a bounded time to land, leave
            if (tid == 0) {
                atomicOr(&st->timeout, 1);
                // the last copy issued into each slot (earlier phases of a slot have completed)
                for (int q = max(i0 - 1, issued - (L::RING - 1)); q <= issued; ++q) {
                    const int k = q - i0 + 1 + kb;
                    unsigned long long* bar = &bars[k % L::RING];
                    for (long long it = 0; it <= kTmaWaitLimit && !mbar_try_wait(bar, (unsigned)((k / L::RING) & 1));
                         ++it) {
                    }
                }
            }
            __syncthreads();
            return false;
        }
        if (DM == 1 && __syncthreads_or(dbad != 0)) return true;
        if (errkey != ERR_NONE) atomicMin(&st->err_key, errkey);
        block_reduce_dd<5>(acc, clipped, sdd, scnt);
        if (tid == 0) {
            StepPartial& out = partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)];
            for (int q = 0; q < 5; ++q) { out.s[q][0] = acc[q].hi; out.s[q][1] = acc[q].lo; }
            out.clipped = clipped;
            out.redo = 0;
        }
        return false;
    }

    // The CTA's chunk. In the drop-in form a chunk whose numerators left the
    // exact-division range is marched a second time with every quotient exact
    // (IEEE division for those), rewriting its trial values, before keys and
    // partials are published; the second march stages its planes after the
    // i1 - i0 + 2 copies of the first, all of which the first has waited for.
    __device__ static void run(const StepParams& P, const CUtensorMap* m_int, const CUtensorMap* m_row,
                               const CUtensorMap* m_col, const CUtensorMap* m_crn, const double* __restrict__ o,
                               const double* __restrict__ cr, const double* __restrict__ p, double* __restrict__ on,
                               double* __restrict__ crn, double* __restrict__ pn, double* __restrict__ eta_next,
                               StepPartial* __restrict__ partials, Status* st) {
        // the staging ring's mbarriers: one array for both marches (declared in
        // a march, each instantiation would have its own)
        __shared__ unsigned long long bars[L::RING];
        if (FAST) {
            run_body<0>(P, m_int, m_row, m_col, m_crn, o, cr, p, on, crn, pn, eta_next, partials, st, bars, 0);
        } else if (run_body<1>(P, m_int, m_row, m_col, m_crn, o, cr, p, on, crn, pn, eta_next, partials, st, bars,
                               0)) {
            const int i0 = blockIdx.z * P.xchunk, i1 = min(P.g.nx, i0 + P.xchunk);
            __syncthreads();
            run_body<2>(P, m_int, m_row, m_col, m_crn, o, cr, p, on, crn, pn, eta_next, partials, st, bars,
                        i1 - i0 + 2);
        }
    }
};

template <bool FAST, int N, int MODE>
__global__ void __launch_bounds__(FTA * FTB, 1)
k_step_fused(const StepParams P, const __grid_constant__ CUtensorMap m_int, const __grid_constant__ CUtensorMap m_row,
             const __grid_constant__ CUtensorMap m_col, const __grid_constant__ CUtensorMap m_crn,
             const double* __restrict__ o, const double* __restrict__ cr, const double* __restrict__ p,
             double* __restrict__ on, double* __restrict__ crn, double* __restrict__ pn,
             double* __restrict__ eta_next, StepPartial* __restrict__ partials, Status* st) {
    OnePassStep<FAST, N, MODE>::run(P, &m_int, &m_row, &m_col, &m_crn, o, cr, p, on, crn, pn, eta_next, partials, st);
}

// The flag combination k_step_fused instantiates with the flags folded (MODE 1).
inline bool fused_common_mode(const StepParams& P) { return P.o_on && P.ck == 0 && P.bounds == 1; }

// Whether the fused step serves grid g with n eta fields (the eta buffer's
// 16-byte alignment is checked at launch).
inline bool fused_step_applies(const Grid& g, int n) {
    return g.dim == 3 && n >= 1 && n <= kFusedMaxEta && g.na % FTA == 0 && g.nb % FTB == 0 && g.nx >= 2;
}

template <bool FAST, int N>
static bool launch_step_fused_n(const StepParams& P, const double* o, const double* cr, const double* p,
                                const double* eta, double* on, double* crn, double* pn, double* eta_next,
                                StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out) {
    const Grid& g = P.g;
    CUtensorMap mi, mr, mc, mk;
    if (!encode_eta_map(&mi, g, N, eta, FTB, FTA, 1) || !encode_eta_map(&mr, g, N, eta, FTB, 1, 1) ||
        !encode_eta_map(&mc, g, N, eta, 2, FTA, 1) || !encode_eta_map(&mk, g, N, eta, 2, 1, N))
        return false;
    using L = FusedLayout<N>;
    const dim3 grid(g.nb / FTB, g.na / FTA, (g.nx + P.xchunk - 1) / P.xchunk);
    if (fused_common_mode(P)) {
        ensure_smem_attr((const void*)k_step_fused<FAST, N, 1>, (int)L::BYTES);
        k_step_fused<FAST, N, 1><<<grid, dim3(FTB, FTA), L::BYTES, stream>>>(P, mi, mr, mc, mk, o, cr, p, on, crn,
                                                                            pn, eta_next, partials, st);
    } else {
        ensure_smem_attr((const void*)k_step_fused<FAST, N, 0>, (int)L::BYTES);
        k_step_fused<FAST, N, 0><<<grid, dim3(FTB, FTA), L::BYTES, stream>>>(P, mi, mr, mc, mk, o, cr, p, on, crn,
                                                                            pn, eta_next, partials, st);
    }
    if (nblocks_out) *nblocks_out = (int)(grid.x * grid.y * grid.z);
    return true;
}

// Launches the fused step for n eta fields; false (nothing launched) when the
// grid, the field count or the buffer alignment does not allow it.
template <bool FAST>
static bool launch_step_fused_form(const StepParams& P, int n, const double* o, const double* cr, const double* p,
                                   const double* eta, double* on, double* crn, double* pn, double* eta_next,
                                   StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out) {
    if (!fused_step_applies(P.g, n) || P.err_slot >= 0) return false;
    if ((reinterpret_cast<unsigned long long>(eta) & 15ull) != 0) return false;
    switch (n) {
#define NICR_FUSED_STEP_CASE(k) \
    case k: return launch_step_fused_n<FAST, k>(P, o, cr, p, eta, on, crn, pn, eta_next, partials, st, stream, nblocks_out);
        NICR_FUSED_STEP_CASE(1) NICR_FUSED_STEP_CASE(2) NICR_FUSED_STEP_CASE(3) NICR_FUSED_STEP_CASE(4)
        NICR_FUSED_STEP_CASE(5) NICR_FUSED_STEP_CASE(6) NICR_FUSED_STEP_CASE(7) NICR_FUSED_STEP_CASE(8)
#undef NICR_FUSED_STEP_CASE
        default: return false;
    }
}

template <bool FAST>
static void step_fused_prepare(int n) {
    switch (n) {
#define NICR_FUSED_PREP_CASE(k) \
    case k:                                                                                  \
        ensure_smem_attr((const void*)k_step_fused<FAST, k, 0>, (int)FusedLayout<k>::BYTES); \
        ensure_smem_attr((const void*)k_step_fused<FAST, k, 1>, (int)FusedLayout<k>::BYTES); \
        break;
        NICR_FUSED_PREP_CASE(1) NICR_FUSED_PREP_CASE(2) NICR_FUSED_PREP_CASE(3) NICR_FUSED_PREP_CASE(4)
        NICR_FUSED_PREP_CASE(5) NICR_FUSED_PREP_CASE(6) NICR_FUSED_PREP_CASE(7) NICR_FUSED_PREP_CASE(8)
#undef NICR_FUSED_PREP_CASE
        default: break;
    }
}

}  // namespace
}  // namespace nicr
