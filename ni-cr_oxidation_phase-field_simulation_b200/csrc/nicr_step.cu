// Explicit time step of the Ni-Cr phase-field model on sm_100a.
//
// One fused pass per step replaces the reference's refresh() + update loop
// (3S:597-620, 3S:761-826; 2D:412-434, 2D:551-597):
//   ghosts -> mu_O, mu_Cr (7/5-point Laplacians) -> mobilities -> six-face
//   conservative fluxes -> c_O, c_Cr, phi trial values -> legacy Ck -> bounds
// Each CTA owns a rows x columns tile and streams along X (2.5D blocking):
// o and cr are staged in shared memory with a radius-2 halo (mu at a
// neighbour needs its Laplacian), phi and the computed mu/M planes with a
// radius-1 halo. Nothing but the trial fields and per-CTA budget partials is
// written to HBM: mu and M never leave the chip.
//
// The arithmetic is the reference's, operation for operation (nvcc -fmad=false;
// divisions by the run constants dx^2, dx, dt use xdiv, which returns the
// correctly rounded quotient), so the FP64 results are bit-identical. The
// kernels themselves are in nicr_step_impl.cuh; this unit compiles the drop-in
// form, nicr_step_fast.cu the reciprocal form. Ghost semantics:
// Neumann copies in X for o, cr, phi, gb and for the computed mu and M
// (refresh copies mu(1) into the ghost, 3S:613-615), periodic rows/columns.
#include <cstring>

#include "nicr_step_impl.cuh"
#include "nicr_step_fused.cuh"

namespace nicr {

__device__ __noinline__ double ieee_div(double a, double b) { return __ddiv_rn(a, b); }

namespace {
// ----------------------------------------------------------------- eta kernels
// S = sum eta_g^2, pairs = sum_{a<b} eta_a^2 eta_b^2 accumulated as in
// rebuild_eta_mask (3S:497-505), gb = scale * min(1, 16 pairs).
__global__ void k_eta_mask(const StepParams P, int neta, const double* __restrict__ eta,
                           double* __restrict__ gb, double* __restrict__ s2, double* __restrict__ pairs_out,
                           Status* st) {
    const Grid& g = P.g;
    const long long n = (long long)g.nx * g.na * g.nb;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(c % g.nb);
        const long long r = c / g.nb;
        const int row = (int)(r % g.na);
        const int x = (int)(r / g.na);
        const long long idx = (long long)x * g.plane + (long long)row * g.pb + col;
        double S = 0., pairs = 0.;
        for (int q = 0; q < neta; ++q) {
            const double e = __ldg(eta + (long long)q * g.nstore + idx);
            const double sq = e * e;
            pairs += S * sq;
            S += sq;
        }
        s2[idx] = S;
        if (pairs_out) pairs_out[idx] = pairs;
        gb[idx] = P.eta_scale * smin(1., 16. * pairs);
    }
}

// Self-check of xdiv on the device against IEEE division: random numerators
// (all finite bit patterns, values of typical magnitude, signed zeros) and,
// every fifth one, a numerator whose quotient lies within ~2^-104 relative of
// a rounding midpoint. The latter: b's odd mantissa part B, M = delta / B mod
// 2^54 for delta in {-3, -1, 1, 3}, kept when M has 54 bits; then
// B * M = A * 2^54 + delta and A (scaled) / b is next to the midpoint M * 2^-54.
__global__ void k_check_division(DivC d, long long n, unsigned long long seed, unsigned long long* counts) {
    unsigned long long bad = 0, total = 0;
    unsigned long long B = ((unsigned long long)__double_as_longlong(d.b) & 0x000FFFFFFFFFFFFFull) | (1ull << 52);
    while (!(B & 1)) B >>= 1;
    unsigned long long inv = B;   // Newton's iteration for 1 / B modulo 2^64
    for (int k = 0; k < 6; ++k) inv *= 2 - B * inv;
    const unsigned long long m54 = (1ull << 54) - 1;
    inv &= m54;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long x = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1));
        x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
        double a;
        if (i % 97 == 0) {
            a = (i & 1) ? -0.0 : 0.0;
        } else if (i % 5 == 1) {
            const long long delta = ((long long)((x >> 60) & 7) - 4) | 1;
            const unsigned long long M = ((unsigned long long)delta * inv) & m54;
            if (!(M >> 53)) continue;
            // num = B * M - delta as 128 bits (hi:lo); its low 54 bits are zero
            unsigned long long lo = B * M, hi = __umul64hi(B, M);
            const unsigned long long dl = (unsigned long long)delta;
            const unsigned long long nlo = lo - dl;
            hi -= (delta > 0 && nlo > lo) ? 1ull : 0ull;
            hi += (delta < 0 && nlo < lo) ? 1ull : 0ull;
            const unsigned long long A = (hi << 10) | (nlo >> 54);
            a = ldexp((double)A, (int)((x >> 8) % 1600) - 800);
            if (x & 1) a = -a;
        } else if (i & 3) {
            const int e = (int)((x >> 56) % 120) - 60;
            a = ldexp((double)(x >> 11) * (1.0 / 9007199254740992.0) + 0.5, e);
            if (x & 1) a = -a;
        } else {
            a = __longlong_as_double((long long)x);
            if (!isfinite(a)) continue;
        }
        const double q = xdiv(a, d), w = __ddiv_rn(a, d.b);
        bad += __double_as_longlong(q) != __double_as_longlong(w);
        ++total;
    }
    atomicAdd(counts, bad);
    atomicAdd(counts + 1, total);
}

// Step commit: partial sums in block order (deterministic), then the budget is
// advanced only when no trial failed (fields swap only on acceptance, 3S:821).
__device__ __forceinline__ void finalize_body(const StepPartial* __restrict__ partials, int nblocks,
                                              DevBudget* budget, Status* st, int accept_mode) {
    __shared__ DD sdd[32 * 5];
    __shared__ long long scnt[32];
    if (st->failed) return;
    DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    long long clipped = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        for (int q = 0; q < 5; ++q) acc[q] = dd_add(acc[q], DD{partials[b].s[q][0], partials[b].s[q][1]});
        clipped += partials[b].clipped;
    }
    block_reduce_dd<5>(acc, clipped, sdd, scnt);
    if (threadIdx.x == 0) {
        if (st->err_key != ERR_NONE) {
            st->failed = 1;
            st->failed_step = st->steps_done;
            return;
        }
        if (accept_mode == 0) {
            // slots: ckO ckCr clipO clipCr bcO -> budget indices 2 3 4 5 6
            for (int q = 0; q < 5; ++q) {
                DD b{budget->v[2 + q][0], budget->v[2 + q][1]};
                b = dd_add(b, acc[q]);
                budget->v[2 + q][0] = b.hi;
                budget->v[2 + q][1] = b.lo;
            }
            budget->clipped += clipped;
            st->steps_done += 1;
        }
    }
}

__global__ void k_step_finalize(const StepPartial* __restrict__ partials, int nblocks, DevBudget* budget,
                                Status* st, int accept_mode) {
    finalize_body(partials, nblocks, budget, st, accept_mode);
}

// Slab commit: the same reduction; the step's outcome is the failing-trial
// key key_of() returns (thread 0, after every slab's step kernels completed),
// so all slabs decide alike.
template <class KeyFn>
__device__ void slab_finalize(const StepPartial* __restrict__ partials, int nblocks, DevBudget* budget, Status* st,
                              KeyFn key_of) {
    __shared__ DD sdd[32 * 5];
    __shared__ long long scnt[32];
    if (st->failed) return;
    DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    long long clipped = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        for (int q = 0; q < 5; ++q) acc[q] = dd_add(acc[q], DD{partials[b].s[q][0], partials[b].s[q][1]});
        clipped += partials[b].clipped;
    }
    block_reduce_dd<5>(acc, clipped, sdd, scnt);
    if (threadIdx.x == 0) {
        const unsigned long long key = key_of();
        if (key != ERR_NONE) {
            st->err_key = key;
            st->failed = 1;
            st->failed_step = st->steps_done;
            return;
        }
        for (int q = 0; q < 5; ++q) {
            DD b{budget->v[2 + q][0], budget->v[2 + q][1]};
            b = dd_add(b, acc[q]);
            budget->v[2 + q][0] = b.hi;
            budget->v[2 + q][1] = b.lo;
        }
        budget->clipped += clipped;
        st->steps_done += 1;
    }
}

// One process: the minimum over every slab's error word of this step, read
// with volatile loads (L2, or the owning GPU's memory for a peer slab).
__global__ void k_step_finalize_slab(const StepPartial* __restrict__ partials, int nblocks, DevBudget* budget,
                                     Status* st, const SlabPeers peers) {
    slab_finalize(partials, nblocks, budget, st, [&]() {
        unsigned long long key = ERR_NONE;
        for (int j = 0; j < peers.n; ++j) {
            const volatile unsigned long long* w = &peers.st[j]->slot_err[peers.slot];
            const unsigned long long v = *w;
            key = v < key ? v : key;
        }
        return key;
    });
}

// One process per slab: the word the ranks reduced with a MIN collective
// (kAgreeNone: every trial passed).
__global__ void k_step_finalize_agreed(const StepPartial* __restrict__ partials, int nblocks, DevBudget* budget,
                                       Status* st, const long long* agreed) {
    slab_finalize(partials, nblocks, budget, st, [&]() {
        const long long v = *(const volatile long long*)agreed;
        return v == kAgreeNone ? ERR_NONE : (unsigned long long)v;
    });
}

// The signed agreement word of this step from the slab's error word.
__global__ void k_agree_word(const Status* st, int slot, long long* agree) {
    const unsigned long long k = st->slot_err[slot];
    *agree = k == ERR_NONE ? kAgreeNone : (long long)k;
}

// Strided runs of double pairs: blockIdx.y picks the segment, the CTAs of a
// row of blocks stride over its rows x n doubles.
__global__ void k_copy_segments(const CopyList L, const Status* st) {
    if (st && st->failed) return;
    const CopySeg& S = L.s[blockIdx.y];
    const long long pairs = S.n / 2, total = pairs * S.rows;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / pairs, c = 2 * (q - r * pairs);
        const double2 v = *reinterpret_cast<const double2*>(S.src + r * S.src_pitch + c);
        *reinterpret_cast<double2*>(S.dst + r * S.dst_pitch + c) = v;
    }
}

// Batched commit: block b commits domain b (same arithmetic as k_step_finalize).
__global__ void k_finalize_batch(const __grid_constant__ FinalizeBatch B) {
    const FinalizeDomain& d = B.d[blockIdx.x];
    finalize_body(d.partials, d.nblocks, d.budget, d.st, 0);
}

// refresh() for output: mu at interior cells, M at interior cells.
template <int DIM>
__global__ void k_refresh(const StepParams P, const double* __restrict__ o, const double* __restrict__ cr,
                          const double* __restrict__ p, const double* __restrict__ gb, double* __restrict__ muO,
                          double* __restrict__ muCr, double* __restrict__ mo, double* __restrict__ mc) {
    const Grid& g = P.g;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = DIM == 3 ? blockIdx.y * blockDim.y + threadIdx.y : 0;
    const int x = blockIdx.z;
    if (col >= g.nb || row >= g.na) return;
    const long long idx = (long long)x * g.plane + (long long)row * g.pb + col;
    const long long ixm = x > 0 ? idx - g.plane : idx, ixp = x < g.nx - 1 ? idx + g.plane : idx;
    const long long rbase = (long long)x * g.plane;
    const long long ibm = rbase + (long long)row * g.pb + (col == 0 ? g.nb - 1 : col - 1);
    const long long ibp = rbase + (long long)row * g.pb + (col == g.nb - 1 ? 0 : col + 1);
    long long iam = idx, iap = idx;
    if (DIM == 3) {
        iam = rbase + (long long)(row == 0 ? g.na - 1 : row - 1) * g.pb + col;
        iap = rbase + (long long)(row == g.na - 1 ? 0 : row + 1) * g.pb + col;
    }
    auto lapf = [&](const double* a) {
        const double c = a[idx];
        if (DIM == 3)
            return xdiv((a[ixp] - 2. * c + a[ixm]), P.v_dxdx) + xdiv((a[iap] - 2. * c + a[iam]), P.v_dada)
                 + xdiv((a[ibp] - 2. * c + a[ibm]), P.v_dbdb);
        return xdiv((a[ixp] - 2. * c + a[ixm]), P.v_dxdx) + xdiv((a[ibp] - 2. * c + a[ibm]), P.v_dbdb);
    };
    const double oc = o[idx], cc = cr[idx];
    const double hh = h(p[idx]);
    muO[idx] = mu_o_local(oc, cc, hh) - 2. * Phys::ko * lapf(o);
    muCr[idx] = mu_cr_local(oc, cc, hh) - 2. * Phys::kc * lapf(cr);
    const double gbv = P.grains ? gb[idx] : 0.;
    mo[idx] = P.o_on ? mobility(oc, hh, gbv, Phys::bmo, Phys::boo, P.gbm1_o) : 0.;
    mc[idx] = mobility(cc, hh, gbv, Phys::bmc, Phys::boc, P.gbm1_cr);
}

}  // namespace

// ----------------------------------------------------------------- launchers
static long long step_tiles(const Grid& g) {
    return g.dim == 3 ? (long long)((g.nb + TB3 - 1) / TB3) * ((g.na + TA3 - 1) / TA3) : (g.nb + TB2 - 1) / TB2;
}
static int forced_xchunk() {
    static int forced = -1;
    if (forced < 0) {
        const char* e = getenv("NICR_XCHUNK");
        forced = e ? std::max(1, atoi(e)) : 0;
    }
    return forced;
}

int choose_xchunk(const Grid& g) {
    return choose_xchunk_batch(&g, 1);
}

int choose_xchunk_fused(const Grid& g) {
    if (forced_xchunk() > 0) return std::min(forced_xchunk(), g.nx);
    const long long tiles = (long long)(g.na / FTA) * (g.nb / FTB), slots = 148;
    int best = g.nx;
    long long best_cost = -1;
    for (int c : xchunk_candidates(g.nx)) {
        const long long ctas = tiles * ((g.nx + c - 1) / c);
        const long long cost = ((ctas + slots - 1) / slots) * (c + 2);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = c; }
    }
    return best;
}

// One chunk for all domains of a batch: the same cost with the CTAs of every
// domain sharing the waves (chunks above a domain's nx clamp to it).
std::vector<int> xchunk_candidates(int nxmax) {
    std::vector<int> cand;
    for (int c = nxmax;; c = (c + 1) / 2) {
        cand.push_back(c);
        if (c == 1) break;
    }
    for (int c = 1; c < nxmax; c *= 2) cand.push_back(c);
    std::sort(cand.begin(), cand.end(), [](int a, int b) { return a > b; });
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    return cand;
}

int choose_xchunk_batch(const Grid* grids, int n) {
    int nxmax = 1;
    bool any3 = false;
    for (int d = 0; d < n; ++d) {
        nxmax = std::max(nxmax, grids[d].nx);
        any3 = any3 || grids[d].dim == 3;
    }
    if (forced_xchunk() > 0) return std::min(forced_xchunk(), nxmax);
    const long long slots = 148LL * (any3 ? 2 : 4);
    const std::vector<int> cand = xchunk_candidates(nxmax);
    int best = nxmax;
    long long best_cost = -1;
    for (int c : cand) {
        long long ctas = 0;
        for (int d = 0; d < n; ++d) ctas += step_tiles(grids[d]) * ((grids[d].nx + c - 1) / c);
        const long long cost = ((ctas + slots - 1) / slots) * (c + 2);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = c; }
    }
    return best;
}

int step_main_blocks(const StepParams& P) {
    const dim3 grid = P.g.dim == 3 ? step_grid<3, TA3, TB3>(P) : step_grid<2, TA2, TB2>(P);
    return (int)(grid.x * grid.y * grid.z);
}

void step_kernels_prepare(const StepParams& P) {
    if (P.fast) {
        step_kernels_prepare_fast(P);
        return;
    }
    if (P.g.dim != 3) return;   // the 2D tile fits the default 48 KB
    using T = Tile<3, TA3, TB3>;
    const bool m3 = step_minb_for(P) == 3;
    const void* k = m3 ? (const void*)k_step_main<3, TA3, TB3, 3, false> : (const void*)k_step_main<3, TA3, TB3, 2, false>;
    ensure_smem_attr(k, (int)T::SMEM_BYTES);
}

int step_main_kernels(const StepParams& P) { return P.fast ? 1 : 2; }

void launch_step_main(const StepParams& P, const double* o, const double* cr, const double* p, const double* gb,
                      const double* s2, double* on, double* crn, double* pn, StepPartial* partials, Status* st,
                      cudaStream_t stream, int* nblocks_out) {
    if (P.fast) launch_step_main_fast(P, o, cr, p, gb, s2, on, crn, pn, partials, st, stream, nblocks_out);
    else launch_step_form<false>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, stream, nblocks_out);
}

bool step_fused_applies(const Grid& g, int neta) { return fused_step_applies(g, neta); }

bool launch_step_fused(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                       const double* eta, double* on, double* crn, double* pn, double* eta_next,
                       StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out) {
    if (P.fast)
        return launch_step_fused_fast(P, neta, o, cr, p, eta, on, crn, pn, eta_next, partials, st, stream,
                                      nblocks_out);
    return launch_step_fused_form<false>(P, neta, o, cr, p, eta, on, crn, pn, eta_next, partials, st, stream,
                                         nblocks_out);
}

void step_fused_prepare(const StepParams& P, int neta) {
    if (P.fast) step_fused_prepare_fast(P, neta);
    else if (fused_step_applies(P.g, neta)) step_fused_prepare<false>(neta);
}

void launch_eta_mask(const StepParams& P, int neta, const double* eta, double* gb, double* s2, double* pairs,
                     Status* st, cudaStream_t stream) {
    const long long n = P.g.ncells;
    const int threads = 256;
    const long long want = (n + threads - 1) / threads;
    const int blocks = (int)(want < 148 * 32 ? want : 148 * 32);
    k_eta_mask<<<blocks, threads, 0, stream>>>(P, neta, eta, gb, s2, pairs, st);
}

void launch_eta_update(const StepParams& P, int neta, const double* eta, const double* s2, const double* p,
                       double* eta_next, double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    if (P.fast) launch_eta_update_fast(P, neta, eta, s2, p, eta_next, gb_next, s2_next, st, stream);
    else launch_eta_form<false>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, st, stream);
}

void launch_step_finalize(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st, int accept_mode,
                          cudaStream_t stream) {
    k_step_finalize<<<1, 256, 0, stream>>>(partials, nblocks, budget, st, accept_mode);
}

void launch_step_finalize_slab(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st,
                               const SlabPeers& peers, cudaStream_t stream) {
    k_step_finalize_slab<<<1, 256, 0, stream>>>(partials, nblocks, budget, st, peers);
}

void launch_step_finalize_agreed(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st,
                                 const long long* agreed, cudaStream_t stream) {
    k_step_finalize_agreed<<<1, 256, 0, stream>>>(partials, nblocks, budget, st, agreed);
}

void launch_agree_word(const Status* st, int slot, long long* agree, cudaStream_t stream) {
    k_agree_word<<<1, 1, 0, stream>>>(st, slot, agree);
}

void launch_copy_segments(const CopyList& L, const Status* st, cudaStream_t stream) {
    if (L.count <= 0) return;
    long long most = 0;
    for (int i = 0; i < L.count; ++i) most = std::max(most, L.s[i].n / 2 * L.s[i].rows);
    const long long want = (most + 255) / 256;
    const int bx = (int)std::max(1LL, std::min(want, 148LL * 4));
    k_copy_segments<<<dim3(bx, L.count), 256, 0, stream>>>(L, st);
}

void launch_finalize_batch(const FinalizeDomain* doms, int n, cudaStream_t stream) {
    for (int i0 = 0; i0 < n; i0 += kFinalizeMax) {
        FinalizeBatch B{};
        B.n = n - i0 < kFinalizeMax ? n - i0 : kFinalizeMax;
        for (int i = 0; i < B.n; ++i) B.d[i] = doms[i0 + i];
        k_finalize_batch<<<B.n, 256, 0, stream>>>(B);
    }
}

// The shared part of a domain's parameters: everything but what BatchSlim carries.
static StepParams slim_base(StepParams sp) {
    sp.g = Grid{};
    sp.layer_o = 0.;
    sp.inlet = 0;
    sp.x_hi = 0;
    sp.key_ncells = 0;
    return sp;
}

// One compact launch for the whole batch when every domain has the same
// dimensionality, form and shared parameters (compared bytewise: the model's
// parameter blocks are value-initialised, padding included); false otherwise.
static bool launch_step_batch_slim(BatchDomain* doms, int n, cudaStream_t stream) {
    if (n > kBatchSlimMax) return false;
    static StepBatchSlim B;   // host staging of the kernel parameters (~27 KB)
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    B.base = doms[0].sp;
    const StepParams ref = slim_base(doms[0].sp);
    for (int i = 0; i < n; ++i) {
        const StepParams b = slim_base(doms[i].sp);
        if (std::memcmp(&b, &ref, sizeof(StepParams)) != 0 || doms[i].sp.x_lo != 0 || doms[i].sp.err_slot >= 0)
            return false;
    }
    const int dim = doms[0].sp.g.dim, fast = doms[0].sp.fast;
    B.n = n;
    int nb = 0;
    for (int i = 0; i < n; ++i) {
        const BatchDomain& d = doms[i];
        const dim3 grid = dim == 3 ? step_grid<3, TA3, TB3>(d.sp) : step_grid<2, TA2, TB2>(d.sp);
        BatchSlim& s = B.d[i];
        s.g = d.sp.g;
        s.layer_o = d.sp.layer_o;
        s.key_ncells = d.sp.key_ncells;
        s.x_hi = d.sp.x_hi;
        s.inlet = d.sp.inlet;
        s.gx = (int)grid.x;
        s.gy = (int)grid.y;
        s.block0 = nb;
        s.pad = 0;
        s.o = d.o; s.cr = d.cr; s.p = d.p; s.gb = d.gb; s.s2 = d.s2;
        s.on = d.on; s.crn = d.crn; s.pn = d.pn;
        s.partials = d.partials;
        s.st = d.st;
        doms[i].nblocks = (int)(grid.x * grid.y * grid.z);
        nb += doms[i].nblocks;
    }
    if (fast) launch_batch_slim_fast(B, nb, dim, stream);
    else if (dim == 3) launch_batch_slim<3, TA3, TB3, 2, false>(B, nb, stream);
    else launch_batch_slim<2, TA2, TB2, 4, false>(B, nb, stream);
    return true;
}

int launch_step_batch(BatchDomain* doms, int n, cudaStream_t stream) {
    if (launch_step_batch_slim(doms, n, stream)) return 1;
    int launches = 0;
    int i = 0;
    while (i < n) {
        // a group: consecutive domains of one dimensionality and form, at most kBatchMax
        StepBatch B{};
        const int dim = doms[i].sp.g.dim, fast = doms[i].sp.fast;
        int nb = 0;
        while (i < n && B.n < kBatchMax && doms[i].sp.g.dim == dim && doms[i].sp.fast == fast) {
            BatchDomain d = doms[i];
            const dim3 grid = dim == 3 ? step_grid<3, TA3, TB3>(d.sp) : step_grid<2, TA2, TB2>(d.sp);
            d.gx = (int)grid.x;
            d.gy = (int)grid.y;
            d.block0 = nb;
            nb += (int)(grid.x * grid.y * grid.z);
            doms[i].nblocks = (int)(grid.x * grid.y * grid.z);
            B.d[B.n++] = d;
            ++i;
        }
        if (fast) launch_batch_group_fast(B, nb, dim, stream);
        else if (dim == 3) launch_batch_group<3, TA3, TB3, 2, false>(B, nb, stream);
        else launch_batch_group<2, TA2, TB2, 4, false>(B, nb, stream);
        ++launches;
    }
    return launches;
}

void launch_refresh(const StepParams& P, const double* o, const double* cr, const double* p, const double* gb,
                    double* muO, double* muCr, double* mo, double* mc, cudaStream_t stream) {
    const Grid& g = P.g;
    if (g.dim == 3) {
        const dim3 block(32, 8);
        const dim3 grid((g.nb + 31) / 32, (g.na + 7) / 8, g.nx);
        k_refresh<3><<<grid, block, 0, stream>>>(P, o, cr, p, gb, muO, muCr, mo, mc);
    } else {
        const dim3 block(128, 1);
        const dim3 grid((g.nb + 127) / 128, 1, g.nx);
        k_refresh<2><<<grid, block, 0, stream>>>(P, o, cr, p, gb, muO, muCr, mo, mc);
    }
}

long long check_division(double b, long long n, unsigned long long seed, long long* tested) {
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess) return -1;
    cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    k_check_division<<<148 * 8, 256>>>(make_divc(b), n, seed, d);
    unsigned long long h[2] = {0, 0};
    const cudaError_t e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return -1;
    if (tested) *tested = (long long)h[1];
    return (long long)h[0];
}

}  // namespace nicr
