// Ordered Ksp nucleation (Model::nucleate / valid_nucleus / stamp,
// 3S:687-724, 3S:752-759; 2D:493-516, 2D:543-550) on the GPU.
//
// The reference scans cells in (i,j,k) order and stamps a hard oxide ball at
// every cell that (on the state as modified by the earlier stamps of the same
// scan) has phi <= .01, o*cr > Ksp and no cell with phi > .01 closer than
// r + gap. Stamps only raise phi (to 1, in cells that had phi < .01), so:
//   * a cell that fails the test on the pre-scan state fails it later too;
//   * a pre-scan candidate c is stamped iff it was not itself stamped earlier
//     in the scan and no cell stamped earlier lies within r + gap of it.
// Pass 1 (parallel) evaluates the pre-scan test for every cell; pass 2 compacts
// the candidates in reference order; pass 3 (one CTA) walks them in order,
// stamps accepted balls, and marks every cell within r + gap of a stamped cell
// in a "blocked" map (exact: the marked set is the Minkowski sum of the
// stamped cells and the exclusion ball, precomputed as integer offsets).
// Distances are integer-valued: 3D compares sqrt(D) < r + gap with IEEE sqrt
// like the reference; 2D uses the reference's C-library hypot, tabulated on
// the host for the integer offsets that occur.
#include <cmath>
#include <cuda_runtime.h>
#include "nicr_kernels.h"
#include "nicr_ksp.h"
#include "nicr_physics.h"

namespace nicr {

namespace {

struct AxisNb {
    int count, lo0, hi0, lo1, hi1;
};
// periodic_neighborhood (3S:220-231)
__device__ __forceinline__ int bounded_reach(double radius, int n) { return radius >= n ? n : (int)ceil(radius); }
__device__ AxisNb periodic_nb(int center, double radius, int n) {
    const int r = bounded_reach(radius, n);
    AxisNb a{0, 0, 0, 0, 0};
    if (2LL * r + 1 >= n) { a.count = 1; a.lo0 = 1; a.hi0 = n; return a; }
    const long long lo = (long long)center - r, hi = (long long)center + r;
    if (lo < 1) { a.count = 2; a.lo0 = 1; a.hi0 = (int)hi; a.lo1 = (int)(lo + n); a.hi1 = n; }
    else if (hi > n) { a.count = 2; a.lo0 = 1; a.hi0 = (int)(hi - n); a.lo1 = (int)lo; a.hi1 = n; }
    else { a.count = 1; a.lo0 = (int)lo; a.hi0 = (int)hi; }
    return a;
}

__device__ __forceinline__ long long gidx(const KspDev& K, int i1, int j1, int k1) {
    // 1-based domain indices -> device index of the stored plane i1-1-x_off.
    // 3D: (i,j,k); 2D: (i,j) with j the column.
    const Grid& g = K.g;
    if (g.dim == 3) return (long long)(i1 - 1 - K.x_off) * g.plane + (long long)(j1 - 1) * g.pb + (k1 - 1);
    return (long long)(i1 - 1 - K.x_off) * g.plane + (j1 - 1);
}
// stored plane of domain index i1, or -1 when this domain/slab does not store it
__device__ __forceinline__ int stored_plane(const KspDev& K, int i1) {
    const int li = i1 - 1 - K.x_off;
    return li >= 0 && li < K.g.nx ? li : -1;
}

// valid_nucleus on the pre-scan state (3S:687-703, 2D:493-502)
__device__ bool valid_prescan(const KspDev& K, const double* __restrict__ p, int x, int y, int z) {
    const Grid& g = K.g;
    const double r = K.radius;
    if (x - r < 5. || x + r > (double)(K.nx - 3)) return false;
    const double limit = r + K.gap;
    if (g.dim == 2) {
        const int sr = (int)ceil(r + K.gap);
        const int i0 = max(1, x - sr), i1 = min(K.nx, x + sr);
        for (int i = i0; i <= i1; ++i)
            for (int j = 1; j <= K.ny; ++j) {
                if (__ldg(p + gidx(K, i, j, 0)) > .01) {
                    const int dj = (int)min_image((double)(j - y), (double)K.ny);
                    if (K.hyp2d[abs(i - x) * K.hyp_stride + abs(dj)]) return false;
                }
            }
        return true;
    }
    const AxisNb ys = periodic_nb(y, limit, K.ny), zs = periodic_nb(z, limit, K.nz);
    const int sr = bounded_reach(limit, K.nx);
    const long long a0 = (long long)x - sr, a1 = (long long)x + sr;
    for (int i = (int)(a0 > 1 ? a0 : 1); i <= (int)(a1 < K.nx ? a1 : K.nx); ++i)
        for (int jy = 0; jy < ys.count; ++jy) {
            const int jlo = jy ? ys.lo1 : ys.lo0, jhi = jy ? ys.hi1 : ys.hi0;
            for (int j = jlo; j <= jhi; ++j)
                for (int kz = 0; kz < zs.count; ++kz) {
                    const int klo = kz ? zs.lo1 : zs.lo0, khi = kz ? zs.hi1 : zs.hi0;
                    for (int k = klo; k <= khi; ++k) {
                        if (__ldg(p + gidx(K, i, j, k)) > .01) {
                            const double di = (double)(i - x), dj = min_image((double)(j - y), (double)K.ny),
                                         dk = min_image((double)(k - z), (double)K.nz);
                            if (sqrt(di * di + dj * dj + dk * dk) < limit) return false;
                        }
                    }
                }
        }
    return true;
}

__global__ void k_ksp_candidates(const KspDev K, const double* __restrict__ o, const double* __restrict__ cr,
                                 const double* __restrict__ p, unsigned char* __restrict__ flag, Status* st) {
    if (st->failed) return;
    const Grid& g = K.g;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(c % g.nb);
        const long long r = c / g.nb;
        const int row = (int)(r % g.na);
        const int xi = (int)(r / g.na);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        unsigned char f = 0;
        const double pv = __ldg(p + idx);
        if (xi >= K.x_lo && xi < K.x_hi && pv <= .01 && __ldg(o + idx) * __ldg(cr + idx) > K.ksp) {
            const int x = xi + K.x_off + 1;
            if (g.dim == 3) f = valid_prescan(K, p, x, row + 1, col + 1) ? 1 : 0;
            else f = valid_prescan(K, p, x, col + 1, 0) ? 1 : 0;
        }
        flag[c] = f;
    }
}

// 3D pre-scan test by an exact, separable bounded distance transform instead
// of a search of the (2 reach + 1)^3 exclusion box per candidate (whose cost
// grows with the number of candidates: a supersaturated 256^3 grid has 16.7M).
// valid_prescan rejects a candidate when some cell with phi > .01 lies in its
// box (|di| <= reach in x within [1, nx]; |dj|, |dk| <= reach periodic) at
// sqrt(di^2 + dj^2 + dk^2) < r + gap, with dj, dk minimum-image offsets. The
// least di^2 + dj^2 + dk^2 over the box's occupied cells is computed in three
// passes (z, then y, then x), each the minimum over the axis' offsets of
// offset^2 plus the previous pass' value. Offsets that wrap a short axis twice
// only add larger copies of the minimum-image distance, so the minimum is the
// reference's; the distances are integers, so sqrt of the exact minimum
// decides as the reference's first hit does.
constexpr int kEdtInf = 1 << 29;

__device__ __forceinline__ int wrap_axis(int v, int n) { v %= n; return v < 0 ? v + n : v; }

__global__ void k_ksp_edt_z(const KspDev K, const double* __restrict__ p, int* __restrict__ dz2, int R, Status* st) {
    if (st->failed) return;
    const Grid& g = K.g;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(c % g.nb);
        const long long r = c / g.nb;
        const int row = (int)(r % g.na);
        const int xi = (int)(r / g.na);
        const double* base = p + (long long)xi * g.plane + (long long)row * g.pb;
        int best = kEdtInf;
        for (int d = -R; d <= R; ++d)
            if (__ldg(base + wrap_axis(col + d, g.nb)) > .01) best = min(best, d * d);
        dz2[c] = best;
    }
}

__global__ void k_ksp_edt_y(const KspDev K, const int* __restrict__ dz2, int* __restrict__ dyz2, int R, Status* st) {
    if (st->failed) return;
    const Grid& g = K.g;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(c % g.nb);
        const long long r = c / g.nb;
        const int row = (int)(r % g.na);
        const long long xi = r / g.na;
        int best = kEdtInf;
        for (int d = -R; d <= R; ++d) {
            const int v = __ldg(dz2 + (xi * g.na + wrap_axis(row + d, g.na)) * g.nb + col);
            if (v < kEdtInf) best = min(best, v + d * d);
        }
        dyz2[c] = best;
    }
}

// The x pass with the point test (phi <= .01, o*cr > Ksp, own plane, the
// reference's x-range test): the candidate flags.
__global__ void k_ksp_candidates_edt(const KspDev K, const double* __restrict__ o, const double* __restrict__ cr,
                                     const double* __restrict__ p, const int* __restrict__ dyz2, int R,
                                     unsigned char* __restrict__ flag, Status* st) {
    if (st->failed) return;
    const Grid& g = K.g;
    const double limit = K.radius + K.gap;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(c % g.nb);
        const long long r = c / g.nb;
        const int row = (int)(r % g.na);
        const int xi = (int)(r / g.na);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        unsigned char f = 0;
        const double pv = __ldg(p + idx);
        if (xi >= K.x_lo && xi < K.x_hi && pv <= .01 && __ldg(o + idx) * __ldg(cr + idx) > K.ksp) {
            const int x = xi + K.x_off + 1;
            if (!(x - K.radius < 5. || x + K.radius > (double)(K.nx - 3))) {
                int best = kEdtInf;
                for (int d = -R; d <= R; ++d) {
                    const int xd = x + d, li = xd - 1 - K.x_off;
                    if (xd < 1 || xd > K.nx || li < 0 || li >= g.nx) continue;
                    const int v = __ldg(dyz2 + ((long long)li * g.na + row) * g.nb + col);
                    if (v < kEdtInf) best = min(best, v + d * d);
                }
                f = (best < kEdtInf && sqrt((double)best) < limit) ? 0 : 1;
            }
        }
        flag[c] = f;
    }
}

// Ordered compaction of flagged cells: per-block counts, then ordered writes.
constexpr int CBLK = 256, CITEMS = 16;  // each block covers CBLK*CITEMS cells
__global__ void k_ksp_count(const unsigned char* __restrict__ flag, long long n, int* counts) {
    const long long base = (long long)blockIdx.x * CBLK * CITEMS;
    int cnt = 0;
    for (int q = 0; q < CITEMS; ++q) {
        const long long c = base + (long long)q * CBLK + threadIdx.x;
        if (c < n && flag[c]) ++cnt;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    __shared__ int s[CBLK / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < CBLK / 32; ++w) t += s[w];
        counts[blockIdx.x] = t;
    }
}
__global__ void k_ksp_write(const unsigned char* __restrict__ flag, long long n, const int* __restrict__ counts,
                            long long* __restrict__ list, int* total, int nblocks) {
    __shared__ long long base_s;
    __shared__ int wsum[CBLK / 32];
    if (threadIdx.x == 0) {
        long long b = 0;
        for (int q = 0; q < (int)blockIdx.x; ++q) b += counts[q];
        base_s = b;
        if (blockIdx.x == nblocks - 1) *total = (int)(b + counts[blockIdx.x]);
    }
    __syncthreads();
    long long running = base_s;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long base = (long long)blockIdx.x * CBLK * CITEMS;
    for (int q = 0; q < CITEMS; ++q) {
        const long long c = base + (long long)q * CBLK + threadIdx.x;
        const bool f = c < n && flag[c];
        const unsigned ball = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wsum[w] = __popc(ball);
        __syncthreads();
        int before = 0, tot = 0;
        for (int ww = 0; ww < CBLK / 32; ++ww) { if (ww < w) before += wsum[ww]; tot += wsum[ww]; }
        if (f) list[running + before + __popc(ball & ((1u << lane) - 1u))] = c;
        running += tot;
        __syncthreads();
    }
}

// stamp(x,y,z) (3S:704-724 / 2D:503-516) on the stored cells: ball cells with
// phi < .01 become oxide. nucO/nucCr collect the increments of the own planes
// (a slab's halo planes are stamped too but counted by their owner). Returns
// the number of cells this thread set.
__device__ int stamp_ball(const KspDev& K, int x, int y, int z, double* o, double* cr, double* p, double* eta,
                          DD& nucO, DD& nucCr) {
    const Grid& g = K.g;
    const int tid = threadIdx.x;
    int cells = 0;
    const double r2 = K.radius * K.radius;
    const long long lo = (long long)K.x_off + 1, hi = (long long)K.x_off + g.nx;   // stored domain planes
    auto set_cell = [&](long long idx, int i) {
        const int li = i - 1 - K.x_off;
        if (li >= K.x_lo && li < K.x_hi) {
            nucO = dd_add(nucO, Phys::oxideO - o[idx]);
            nucCr = dd_add(nucCr, Phys::oxideCr - cr[idx]);
        }
        o[idx] = Phys::oxideO; cr[idx] = Phys::oxideCr; p[idx] = 1.;
        for (int e = 0; e < K.neta; ++e) eta[(long long)e * g.nstore + idx] = 0.;
        ++cells;
    };
    if (g.dim == 3) {
        const int rr = bounded_reach(K.radius, K.nx);
        const AxisNb ys = periodic_nb(y, K.radius, K.ny), zs = periodic_nb(z, K.radius, K.nz);
        const int i0 = (int)max(lo, max(1LL, (long long)x - rr)), i1 = (int)min(hi, min((long long)K.nx, (long long)x + rr));
        if (i1 < i0) return 0;
        const int ny_n = (ys.hi0 - ys.lo0 + 1) + (ys.count > 1 ? ys.hi1 - ys.lo1 + 1 : 0);
        const int nz_n = (zs.hi0 - zs.lo0 + 1) + (zs.count > 1 ? zs.hi1 - zs.lo1 + 1 : 0);
        const long long tot = (long long)(i1 - i0 + 1) * ny_n * nz_n;
        for (long long q = tid; q < tot; q += blockDim.x) {
            const int kq = (int)(q % nz_n);
            const long long t = q / nz_n;
            const int jq = (int)(t % ny_n);
            const int i = i0 + (int)(t / ny_n);
            const int n0y = ys.hi0 - ys.lo0 + 1, n0z = zs.hi0 - zs.lo0 + 1;
            const int j = jq < n0y ? ys.lo0 + jq : ys.lo1 + (jq - n0y);
            const int k = kq < n0z ? zs.lo0 + kq : zs.lo1 + (kq - n0z);
            const double dy = min_image((double)(j - y), (double)K.ny), dz = min_image((double)(k - z), (double)K.nz);
            const long long idx = gidx(K, i, j, k);
            if ((double)((i - x) * (i - x)) + dy * dy + dz * dz <= r2 && p[idx] < .01) set_cell(idx, i);
        }
    } else {
        const int rr = (int)ceil(K.radius);
        const int i0 = (int)max(lo, (long long)max(1, x - rr)), i1 = (int)min(hi, (long long)min(K.nx, x + rr));
        if (i1 < i0) return 0;
        const long long tot = (long long)(i1 - i0 + 1) * K.ny;
        for (long long q = tid; q < tot; q += blockDim.x) {
            const int j = (int)(q % K.ny) + 1;
            const int i = i0 + (int)(q / K.ny);
            const double dy = min_image((double)(j - y), (double)K.ny);
            const long long idx = gidx(K, i, j, 0);
            if ((double)((i - x) * (i - x)) + dy * dy <= r2 && p[idx] < .01) set_cell(idx, i);
        }
    }
    return cells;
}

// Exclusion marks of a stamped nucleus for the later candidates of the scan,
// on the stored cells. full: the stamp set the whole ball, whose marks are the
// precomputed shadow (Minkowski sum of the ball and the exclusion ball);
// otherwise (some ball cell had phi == .01 exactly) every cell of the
// exclusion box is tested against the ball cells that are oxide now.
__device__ void mark_excluded(const KspDev& K, int x, int y, int z, bool full, const double* p,
                              unsigned char* blocked, KspResult* res, bool count_partial) {
    const Grid& g = K.g;
    const int tid = threadIdx.x;
    if (full) {
        for (int q = tid; q < K.n_shadow; q += blockDim.x) {
            const int di = K.shadow[3 * q], dj = K.shadow[3 * q + 1], dk = K.shadow[3 * q + 2];
            const int i = x + di;
            if (i < 1 || i > K.nx) continue;
            const int li = stored_plane(K, i);
            if (li < 0) continue;
            if (g.dim == 3) {
                const int j = ((y - 1 + dj) % K.ny + K.ny) % K.ny;
                const int k = ((z - 1 + dk) % K.nz + K.nz) % K.nz;
                blocked[((long long)li * K.ny + j) * K.nz + k] = 1;
            } else {
                const int j = ((y - 1 + dj) % K.ny + K.ny) % K.ny;
                blocked[(long long)li * K.ny + j] = 1;
            }
        }
        return;
    }
    if (count_partial && tid == 0) res->partial_stamps += 1;
    const int R = K.box_half;
    const long long side = 2LL * R + 1;
    const long long tot = g.dim == 3 ? side * side * side : side * side;
    for (long long q = tid; q < tot; q += blockDim.x) {
        int di, dj, dk = 0;
        if (g.dim == 3) { dk = (int)(q % side) - R; dj = (int)((q / side) % side) - R; di = (int)(q / (side * side)) - R; }
        else { dj = (int)(q % side) - R; di = (int)(q / side) - R; }
        const int i = x + di;
        if (i < 1 || i > K.nx) continue;
        const int li = stored_plane(K, i);
        if (li < 0) continue;
        const int jw = ((y - 1 + dj) % K.ny + K.ny) % K.ny + 1;
        const int kw = g.dim == 3 ? ((z - 1 + dk) % K.nz + K.nz) % K.nz + 1 : 0;
        bool hit = false;
        for (int b = 0; b < K.n_ball && !hit; ++b) {
            const int si = x + K.ball[3 * b];
            if (si < 1 || si > K.nx || stored_plane(K, si) < 0) continue;
            const int sj = ((y - 1 + K.ball[3 * b + 1]) % K.ny + K.ny) % K.ny + 1;
            const int sk = g.dim == 3 ? ((z - 1 + K.ball[3 * b + 2]) % K.nz + K.nz) % K.nz + 1 : 0;
            if (p[gidx(K, si, sj, sk)] != 1.) continue;   // not (newly) oxide
            const int ddi = si - i;
            const int ddj = (int)min_image((double)(sj - jw), (double)K.ny);
            if (g.dim == 3) {
                const int ddk = (int)min_image((double)(sk - kw), (double)K.nz);
                hit = sqrt((double)ddi * ddi + (double)ddj * ddj + (double)ddk * ddk) < K.radius + K.gap;
            } else {
                hit = K.hyp2d[abs(ddi) * K.hyp_stride + abs(ddj)] != 0;
            }
        }
        if (hit) {
            if (g.dim == 3) blocked[((long long)li * K.ny + (jw - 1)) * K.nz + (kw - 1)] = 1;
            else blocked[(long long)li * K.ny + (jw - 1)] = 1;
        }
    }
}

// One CTA: ordered greedy resolve + stamps + exclusion marks.
//   mode 0  scan: the nuclei in pre (accepted earlier in the scan by slabs
//           before this one along X: stamps and marks), then the own
//           candidates in order; accepted nuclei go to out (when given)
//   mode 1  one forced stamp at (fx, fy, fz) (Model::stamp)
//   mode 2  the stamps of the nuclei in pre only (no marks, no candidates)
__global__ void __launch_bounds__(1024) k_ksp_resolve(const KspDev K, const long long* __restrict__ list,
                                                      const int* __restrict__ total, int mode, int fx, int fy,
                                                      int fz, const KspNucleus* __restrict__ pre, int npre,
                                                      KspNucleus* out, int cap, double* o, double* cr, double* p,
                                                      double* eta, unsigned char* blocked, DevBudget* budget,
                                                      KspResult* res, Status* st) {
    if (st->failed) return;
    __shared__ long long s_cand;
    __shared__ int s_next;
    __shared__ int s_first[32];
    __shared__ DD s_dd[32][2];
    __shared__ int s_cnt[32];
    const Grid& g = K.g;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const bool forced = mode == 1;
    DD nucO{0., 0.}, nucCr{0., 0.};
    for (int q = 0; q < npre; ++q) {
        const KspNucleus nu = pre[q];
        stamp_ball(K, nu.x, nu.y, nu.z, o, cr, p, eta, nucO, nucCr);
        __syncthreads();
        if (mode == 0) mark_excluded(K, nu.x, nu.y, nu.z, nu.full != 0, p, blocked, res, false);
        __syncthreads();
    }
    const int n = mode == 2 ? 0 : (forced ? 1 : *total);
    int pos = 0, accepted = 0, last_cells = 0, listed = 0;
    const int nw = (int)(blockDim.x >> 5);
    while (mode != 2) {
        // the whole CTA looks at the next blockDim.x candidates from pos; the
        // first (lowest index) that is neither excluded nor stamped since the
        // pre-scan is the next nucleus
        int found = -1;
        if (forced) {
            found = pos < n ? 0 : -1;
        } else {
            while (pos < n) {
                const int q = pos + tid;
                bool ok = false;
                if (q < n) {
                    const long long cq = list[q];
                    const int col = (int)(cq % g.nb);
                    const long long rr = cq / g.nb;
                    const int row = (int)(rr % g.na);
                    const int xi = (int)(rr / g.na);
                    const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
                    ok = !blocked[cq] && p[idx] <= .01;
                }
                const unsigned b = __ballot_sync(0xffffffffu, ok);
                if (lane == 0) s_first[w] = b ? w * 32 + __ffs(b) - 1 : 0x7fffffff;
                __syncthreads();
                if (w == 0) {
                    int v = lane < nw ? s_first[lane] : 0x7fffffff;
                    for (int off = 16; off > 0; off >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, off));
                    if (lane == 0) s_next = v;
                }
                __syncthreads();
                const int first = s_next;
                __syncthreads();   // s_first and s_next are rewritten in the next round
                if (first != 0x7fffffff) {
                    found = pos + first;
                    break;
                }
                pos += (int)blockDim.x;
            }
        }
        if (tid == 0) s_cand = found >= 0 ? (forced ? -1 : list[found]) : -1;
        __syncthreads();
        if (found < 0) break;
        pos = found + 1;
        int x, y, z = 0;
        if (forced) { x = fx; y = fy; z = fz; }
        else {
            const long long cq = s_cand;
            const int col = (int)(cq % g.nb);
            const long long rr = cq / g.nb;
            const int row = (int)(rr % g.na);
            x = (int)(rr / g.na) + 1 + K.x_off;
            if (g.dim == 3) { y = row + 1; z = col + 1; } else { y = col + 1; }
        }
        int cells = stamp_ball(K, x, y, z, o, cr, p, eta, nucO, nucCr);
        for (int off = 16; off > 0; off >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, off);
        if (lane == 0) s_cnt[w] = cells;
        __syncthreads();
        int changed = 0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) changed += s_cnt[ww];
        if (changed) {
            ++accepted;
            if (!forced) {
                if (tid == 0 && out && listed < cap) out[listed] = KspNucleus{x, y, z, changed == K.full_ball ? 1 : 0};
                ++listed;
            }
        }
        last_cells = changed;
        // exclusion marks for the later candidates of this scan
        if (changed && !forced) mark_excluded(K, x, y, z, changed == K.full_ball, p, blocked, res, true);
        __syncthreads();
        if (forced) break;
    }
    // budget: nucO, nucCr, nuclei
    for (int off = 16; off > 0; off >>= 1) {
        nucO = dd_add(nucO, DD{__shfl_down_sync(0xffffffffu, nucO.hi, off), __shfl_down_sync(0xffffffffu, nucO.lo, off)});
        nucCr = dd_add(nucCr, DD{__shfl_down_sync(0xffffffffu, nucCr.hi, off), __shfl_down_sync(0xffffffffu, nucCr.lo, off)});
    }
    if (lane == 0) { s_dd[w][0] = nucO; s_dd[w][1] = nucCr; }
    __syncthreads();
    if (tid == 0) {
        DD a = s_dd[0][0], b = s_dd[0][1];
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) { a = dd_add(a, s_dd[ww][0]); b = dd_add(b, s_dd[ww][1]); }
        DD bo{budget->v[0][0], budget->v[0][1]}, bc{budget->v[1][0], budget->v[1][1]};
        bo = dd_add(bo, a); bc = dd_add(bc, b);
        budget->v[0][0] = bo.hi; budget->v[0][1] = bo.lo;
        budget->v[1][0] = bc.hi; budget->v[1][1] = bc.lo;
        budget->nuclei += accepted;
        if (mode != 2) {
            res->nuclei = accepted;
            res->last_cells = last_cells;
            res->candidates = n;
            res->listed = listed;
        }
    }
}

int cgrid(long long n, int threads, int cap) {
    const long long want = (n + threads - 1) / threads;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

int ksp_compact_blocks(long long ncells) { return (int)((ncells + CBLK * CITEMS - 1) / (CBLK * CITEMS)); }

void launch_ksp_candidates(const KspDev& K, const double* o, const double* cr, const double* p, KspWork& W,
                           Status* st, cudaStream_t stream) {
    const long long n = K.g.ncells;
    cudaMemsetAsync(W.blocked, 0, (size_t)n, stream);
    if (K.g.dim == 3) {
        // the two distance arrays live in the candidate list's storage (8 bytes
        // per cell), which the compaction below overwrites afterwards
        int* dz2 = reinterpret_cast<int*>(W.list);
        int* dyz2 = dz2 + n;
        const double limit = K.radius + K.gap;
        auto reach = [&](int m) { return limit >= m ? m : (int)std::ceil(limit); };
        const int blocks = cgrid(n, 256, 148 * 16);
        k_ksp_edt_z<<<blocks, 256, 0, stream>>>(K, p, dz2, reach(K.nz), st);
        k_ksp_edt_y<<<blocks, 256, 0, stream>>>(K, dz2, dyz2, reach(K.ny), st);
        k_ksp_candidates_edt<<<blocks, 256, 0, stream>>>(K, o, cr, p, dyz2, reach(K.nx), W.flag, st);
    } else {
        k_ksp_candidates<<<cgrid(n, 128, 148 * 64), 128, 0, stream>>>(K, o, cr, p, W.flag, st);
    }
    const int nb = ksp_compact_blocks(n);
    k_ksp_count<<<nb, CBLK, 0, stream>>>(W.flag, n, W.counts);
    k_ksp_write<<<nb, CBLK, 0, stream>>>(W.flag, n, W.counts, W.list, W.total, nb);
}

void launch_ksp_scan(const KspDev& K, double* o, double* cr, double* p, double* eta, KspWork& W, DevBudget* budget,
                     KspResult* res, Status* st, cudaStream_t stream) {
    launch_ksp_candidates(K, o, cr, p, W, st, stream);
    k_ksp_resolve<<<1, 1024, 0, stream>>>(K, W.list, W.total, 0, 0, 0, 0, nullptr, 0, nullptr, 0, o, cr, p, eta,
                                          W.blocked, budget, res, st);
}

void launch_ksp_stamp(const KspDev& K, int x, int y, int z, double* o, double* cr, double* p, double* eta,
                      KspWork& W, DevBudget* budget, KspResult* res, Status* st, cudaStream_t stream) {
    k_ksp_resolve<<<1, 1024, 0, stream>>>(K, W.list, W.total, 1, x, y, z, nullptr, 0, nullptr, 0, o, cr, p, eta,
                                          W.blocked, budget, res, st);
}

void launch_ksp_resolve_slab(const KspDev& K, const KspNucleus* pre, int npre, KspNucleus* out, int cap, double* o,
                             double* cr, double* p, double* eta, KspWork& W, DevBudget* budget, KspResult* res,
                             Status* st, cudaStream_t stream) {
    k_ksp_resolve<<<1, 1024, 0, stream>>>(K, W.list, W.total, 0, 0, 0, 0, pre, npre, out, cap, o, cr, p, eta,
                                          W.blocked, budget, res, st);
}

void launch_ksp_apply(const KspDev& K, const KspNucleus* list, int n, double* o, double* cr, double* p, double* eta,
                      KspWork& W, DevBudget* budget, KspResult* res, Status* st, cudaStream_t stream) {
    if (n <= 0) return;
    k_ksp_resolve<<<1, 1024, 0, stream>>>(K, W.list, W.total, 2, 0, 0, 0, list, n, nullptr, 0, o, cr, p, eta,
                                          W.blocked, budget, res, st);
}

}  // namespace nicr
