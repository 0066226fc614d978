// Initialisation and diagnostics kernels.
//   init_fields   Model constructor field values (3S:362-369)
//   voronoi3      nearest-seed labels + bisector distance, O(cells * seeds * 9)
//                 (3S:450-466; the Gaussian exp of the mask is applied on the
//                 host with the C library, exactly as the reference evaluates it)
//   eta_dist3     competitor distances for the eta initial weights (3S:469-494)
//   center_seed   centre sphere/disc (3S:725-751, 2D:517-542)
//   diagnostics   sums / extrema of Model::log (3S:963-977)
#include <cuda_runtime.h>
#include <math_constants.h>
#include "nicr_kernels.h"
#include "nicr_physics.h"

namespace nicr {

namespace {

__device__ __forceinline__ DD shfl_dd(DD v, int off) {
    return DD{__shfl_down_sync(0xffffffffu, v.hi, off), __shfl_down_sync(0xffffffffu, v.lo, off)};
}

// cell (x,row,col) of a linear interior index in reference order
__device__ __forceinline__ void decode(const Grid& g, long long c, int& x, int& row, int& col) {
    col = (int)(c % g.nb);
    const long long r = c / g.nb;
    row = (int)(r % g.na);
    x = (int)(r / g.na);
}

__global__ void k_init_fields(const InitParams I, double* o, double* cr, double* p) {
    const Grid& g = I.g;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int x, row, col;
        decode(g, c, x, row, col);
        const long long idx = (long long)x * g.plane + (long long)row * g.pb + col;
        double ov = Phys::bulkO, cv = I.bulk_cr;
        if (I.inlet_layer && x + I.x_off == 0) { ov = I.layer_o; cv = Phys::layerCr; }
        o[idx] = ov; cr[idx] = cv; p[idx] = 0.;
    }
}

// competitor_distance (3S:395-406) for seed g against owner
__device__ __forceinline__ double competitor_distance(const double* s, int g, int owner, double x, double y,
                                                      double z, double oY, double oZ, double rbest, int ny, int nz) {
    double db = CUDART_INF;
    const double sx = s[3 * g], sy = s[3 * g + 1], sz = s[3 * g + 2], ox = s[3 * owner];
    for (int im = -1; im <= 1; ++im)
        for (int jm = -1; jm <= 1; ++jm) {
            const double gy = sy + (double)(im * ny), gz = sz + (double)(jm * nz);
            const double ax = sx - x, ay = gy - y, az = gz - z;
            const double rs = ax * ax + ay * ay + az * az;
            const double bx = sx - ox, by = gy - oY, bz = gz - oZ;
            const double sep = sqrt(bx * bx + by * by + bz * bz);
            if (sep > 1.e-14) db = smin(db, smax(0., (rs - rbest) / (2. * sep)));
        }
    return db;
}

// STAGED: the seed table is copied to shared memory (when it fits, up to
// ~8,500 seeds); otherwise the threads read it from global memory (L1/L2).
template <bool STAGED>
__global__ void k_voronoi3(const InitParams I, const double* __restrict__ seeds, double* grain, double* dbout,
                           int* volumes, int* competitor) {
    extern __shared__ double seed_smem[];
    const double* ss = seeds;
    if (STAGED) {
        for (int q = threadIdx.x; q < 3 * I.ng; q += blockDim.x) seed_smem[q] = seeds[q];
        __syncthreads();
        ss = seed_smem;
    }
    const Grid& g = I.g;
    const int ny = g.na, nz = g.nb;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const double x = (xi + I.x_off + 1) - .5, y = (row + 1) - .5, z = (col + 1) - .5;
        int owner = 0;
        double rbest = CUDART_INF, oY = 0., oZ = 0.;
        for (int s = 0; s < I.ng; ++s) {
            const double yy = min_image(ss[3 * s + 1] - y, I.nyd), zz = min_image(ss[3 * s + 2] - z, I.nzd);
            const double ax = ss[3 * s] - x;
            const double rr = ax * ax + yy * yy + zz * zz;
            if (rr < rbest) { rbest = rr; owner = s; oY = y + yy; oZ = z + zz; }
        }
        double db = CUDART_INF;
        int near = -1;   // the first competitor attaining db
        for (int s = 0; s < I.ng; ++s)
            if (s != owner) {
                const double d = competitor_distance(ss, s, owner, x, y, z, oY, oZ, rbest, ny, nz);
                if (d < db) near = s;
                db = smin(db, d);
            }
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        grain[idx] = owner + 1;
        dbout[idx] = db;
        if (competitor) competitor[idx] = near;
        if (xi >= I.x_lo && xi < I.x_hi) atomicAdd(volumes + owner, 1);
    }
}

template <bool STAGED>
__global__ void k_eta_dist3(const InitParams I, const double* __restrict__ seeds, const double* __restrict__ grain,
                            double* eta) {
    extern __shared__ double seed_smem[];
    const double* ss = seeds;
    if (STAGED) {
        for (int q = threadIdx.x; q < 3 * I.ng; q += blockDim.x) seed_smem[q] = seeds[q];
        __syncthreads();
        ss = seed_smem;
    }
    const Grid& g = I.g;
    const int ny = g.na, nz = g.nb;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const int owner = (int)grain[idx] - 1;
        const double x = (xi + I.x_off + 1) - .5, y = (row + 1) - .5, z = (col + 1) - .5;
        const double oy = y + min_image(ss[3 * owner + 1] - y, I.nyd), oz = z + min_image(ss[3 * owner + 2] - z, I.nzd);
        const double ax = ss[3 * owner] - x, ay = oy - y, az = oz - z;
        const double rbest = ax * ax + ay * ay + az * az;
        for (int s = 0; s < I.ng; ++s)
            eta[(long long)s * g.nstore + idx] =
                s == owner ? -1. : competitor_distance(ss, s, owner, x, y, z, oy, oz, rbest, ny, nz);
    }
}

// Face adjacency of the Voronoi grains over the stored cells: adj[a*ng+b] = 1
// when a cell of grain a and its +X (stored planes only), +Y or +Z neighbour
// (periodic) belongs to grain b != a.
__global__ void k_grain_adjacency(const InitParams I, const double* __restrict__ grain, unsigned char* adj) {
    const Grid& g = I.g;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const int a = (int)grain[idx] - 1;
        int nb[3];
        nb[0] = xi + 1 < g.nx ? (int)grain[idx + g.plane] - 1 : a;
        nb[1] = (int)grain[(long long)xi * g.plane + (long long)(row + 1 == g.na ? 0 : row + 1) * g.pb + col] - 1;
        nb[2] = (int)grain[(long long)xi * g.plane + (long long)row * g.pb + (col + 1 == g.nb ? 0 : col + 1)] - 1;
        for (int q = 0; q < 3; ++q)
            if (nb[q] != a) {
                adj[(long long)a * I.ng + nb[q]] = 1;
                adj[(long long)nb[q] * I.ng + a] = 1;
            }
    }
}

template <int N>
__device__ void block_reduce(DD (&v)[N], long long& cnt) {
    __shared__ DD sdd[32 * N];
    __shared__ long long scnt[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int off = 16; off > 0; off >>= 1) {
        for (int q = 0; q < N; ++q) v[q] = dd_add(v[q], shfl_dd(v[q], off));
        cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    }
    if (lane == 0) { for (int q = 0; q < N; ++q) sdd[w * N + q] = v[q]; scnt[w] = cnt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < N; ++q) v[q] = sdd[q];
        cnt = scnt[0];
        for (int ww = 1; ww < nw; ++ww) {
            for (int q = 0; q < N; ++q) v[q] = dd_add(v[q], sdd[ww * N + q]);
            cnt += scnt[ww];
        }
    }
}

// centre hard seed: cells with dx^2+dy^2(+dz^2) <= r^2 (fractional centre)
__global__ void k_center_seed(const InitParams I, double cx, double cy, double cz, double r, int neta, double* o,
                              double* cr, double* p, double* eta, StepPartial* partials) {
    const Grid& g = I.g;
    DD acc[2] = {{0., 0.}, {0., 0.}};
    long long cnt = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        // reference indices are 1-based: i = xi+1, (3D) j = row+1, k = col+1; (2D) j = col+1
        const double ddx = (xi + I.x_off + 1) - cx;
        double d2;
        if (g.dim == 3) {
            const double ddy = (row + 1) - cy, ddz = (col + 1) - cz;
            d2 = ddx * ddx + ddy * ddy + ddz * ddz;
        } else {
            const double ddy = (col + 1) - cy;
            d2 = ddx * ddx + ddy * ddy;
        }
        if (d2 <= r * r) {
            const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
            if (xi >= I.x_lo && xi < I.x_hi) {   // halo planes of a slab are stamped, not counted
                acc[0] = dd_add(acc[0], Phys::oxideO - o[idx]);
                acc[1] = dd_add(acc[1], Phys::oxideCr - cr[idx]);
                ++cnt;
            }
            o[idx] = Phys::oxideO; cr[idx] = Phys::oxideCr; p[idx] = 1.;
            for (int q = 0; q < neta; ++q) eta[(long long)q * g.nstore + idx] = 0.;
        }
    }
    block_reduce<2>(acc, cnt);
    if (threadIdx.x == 0) {
        StepPartial& out = partials[blockIdx.x];
        for (int q = 0; q < 5; ++q) { out.s[q][0] = 0.; out.s[q][1] = 0.; }
        out.s[0][0] = acc[0].hi; out.s[0][1] = acc[0].lo;
        out.s[1][0] = acc[1].hi; out.s[1][1] = acc[1].lo;
        out.clipped = cnt;
    }
}

__global__ void k_reduce_partials(const StepPartial* __restrict__ partials, int nblocks, StepPartial* out) {
    DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    long long cnt = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        for (int q = 0; q < 5; ++q) acc[q] = dd_add(acc[q], DD{partials[b].s[q][0], partials[b].s[q][1]});
        cnt += partials[b].clipped;
    }
    block_reduce<5>(acc, cnt);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 5; ++q) { out->s[q][0] = acc[q].hi; out->s[q][1] = acc[q].lo; }
        out->clipped = cnt;
    }
}

// Model::log sums and extrema. Extrema follow std::min/std::max exactly: a
// value replaces the running one only when strictly smaller (larger), so among
// equal values (e.g. 0 and -0) the first in reference loop order is kept; the
// initial values 1 (min) and 0 (max) come first.
struct Ext {
    double v;
    long long i;
};
__device__ __forceinline__ Ext ext_min(Ext a, Ext b) {
    if (b.v < a.v) return b;
    if (a.v < b.v) return a;
    if (a.v == b.v) return a.i <= b.i ? a : b;
    return isnan(a.v) ? b : a;
}
__device__ __forceinline__ Ext ext_max(Ext a, Ext b) {
    if (a.v < b.v) return b;
    if (b.v < a.v) return a;
    if (a.v == b.v) return a.i <= b.i ? a : b;
    return isnan(a.v) ? b : a;
}
__device__ __forceinline__ Ext shfl_ext(Ext e, int off) {
    return Ext{__shfl_down_sync(0xffffffffu, e.v, off), __shfl_down_sync(0xffffffffu, e.i, off)};
}

__global__ void k_diagnostics(const Grid g, const double* __restrict__ o, const double* __restrict__ cr,
                              const double* __restrict__ p, DiagOut* partials) {
    DD acc[4] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    Ext mn[4] = {{1., -1}, {1., -1}, {1., -1}, {1., -1}}, mx[4] = {{0., -1}, {0., -1}, {0., -1}, {0., -1}};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const double ov = o[idx], cv = cr[idx], pv = p[idx];
        acc[0] = dd_add(acc[0], ov);
        acc[1] = dd_add(acc[1], cv);
        acc[2] = dd_add(acc[2], pv);
        acc[3] = dd_add(acc[3], h(pv));
        mn[0] = ext_min(mn[0], Ext{ov, c}); mx[0] = ext_max(mx[0], Ext{ov, c});
        mn[1] = ext_min(mn[1], Ext{cv, c}); mx[1] = ext_max(mx[1], Ext{cv, c});
        mn[2] = ext_min(mn[2], Ext{1. - ov - cv, c});
        mn[3] = ext_min(mn[3], Ext{pv, c}); mx[3] = ext_max(mx[3], Ext{pv, c});
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int q = 0; q < 4; ++q) {
            mn[q] = ext_min(mn[q], shfl_ext(mn[q], off));
            mx[q] = ext_max(mx[q], shfl_ext(mx[q], off));
        }
    __shared__ Ext smn[32][4], smx[32][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) for (int q = 0; q < 4; ++q) { smn[w][q] = mn[q]; smx[w][q] = mx[q]; }
    long long dummy = 0;
    block_reduce<4>(acc, dummy);   // contains the __syncthreads that publishes smn/smx
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < nw; ++ww)
            for (int q = 0; q < 4; ++q) { mn[q] = ext_min(mn[q], smn[ww][q]); mx[q] = ext_max(mx[q], smx[ww][q]); }
        DiagOut& out = partials[blockIdx.x];
        for (int q = 0; q < 4; ++q) {
            out.sum[q][0] = acc[q].hi; out.sum[q][1] = acc[q].lo;
            out.mn[q] = mn[q].v; out.mx[q] = mx[q].v;
            out.mni[q] = mn[q].i; out.mxi[q] = mx[q].i;
        }
    }
}

__global__ void k_diag_finalize(const DiagOut* __restrict__ partials, int nblocks, DiagOut* out) {
    if (threadIdx.x != 0) return;
    DiagOut r = partials[0];
    for (int b = 1; b < nblocks; ++b) {
        for (int q = 0; q < 4; ++q) {
            DD s = dd_add(DD{r.sum[q][0], r.sum[q][1]}, DD{partials[b].sum[q][0], partials[b].sum[q][1]});
            r.sum[q][0] = s.hi; r.sum[q][1] = s.lo;
            Ext a = ext_min(Ext{r.mn[q], r.mni[q]}, Ext{partials[b].mn[q], partials[b].mni[q]});
            r.mn[q] = a.v; r.mni[q] = a.i;
            Ext z = ext_max(Ext{r.mx[q], r.mxi[q]}, Ext{partials[b].mx[q], partials[b].mxi[q]});
            r.mx[q] = z.v; r.mxi[q] = z.i;
        }
    }
    *out = r;
}

// ---- grain statistics (Model::grain_log, 3S:566-590; grain_energy 3S:546-565)
// Scalars per block: lo/hi of eta (first-in-order extrema over (cell, g)),
// slo/shi of S, sums of S, (1-h)gb and the energy density (dd), max gb,
// unassigned cells; the dominant-grain cell counts go through integer atomics.
struct GrainPart {
    double sum[3][2];        // S, mask, energy
    Ext lo, hi, slo, shi, gbmax;
    long long unassigned;
};
__global__ void k_grain_scalar(const GrainParams G, const double* __restrict__ eta, const double* __restrict__ s2,
                               const double* __restrict__ p, const double* __restrict__ gb,
                               unsigned long long* __restrict__ cells, GrainPart* parts) {
    const Grid& g = G.g;
    DD acc[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
    Ext lo{1., -1}, hi{0., -1}, slo{CUDART_INF, -1}, shi{0., -1}, gbmax{0., -1};
    long long unassigned = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const double S = s2[idx], pv = p[idx], metal = 1. - h(pv), gbv = gb[idx];
        slo = ext_min(slo, Ext{S, c});
        shi = ext_max(shi, Ext{S, c});
        acc[0] = dd_add(acc[0], S);
        acc[1] = dd_add(acc[1], metal * gbv);
        gbmax = ext_max(gbmax, Ext{gbv, c});
        // current_grain (3S:527-533): eta argmax above 1e-12 in metal (phi < .5)
        int id = 0;
        double best = 1.e-12;
        double pairs = 0., Sr = 0.;
        for (int q = 0; q < G.neta; ++q) {
            const double v = eta[(long long)q * g.nstore + idx];
            lo = ext_min(lo, Ext{v, c * G.neta + q});
            hi = ext_max(hi, Ext{v, c * G.neta + q});
            if (v > best) { best = v; id = q + 1; }
            const double sq = v * v;
            pairs += Sr * sq;
            Sr += sq;
        }
        if (pv >= .5) id = 0;
        if (id) atomicAdd(cells + (id - 1), 1ull);
        else if (pv < .5) ++unassigned;
        // energy density: local terms + forward-face gradients (Neumann X, periodic rows/cols)
        double density = grain_energy_density(S, G.dim == 3 ? pairs : G.pairs[idx], pv, G.W, G.A);
        const long long ixp = idx + g.plane;
        const long long iap = (long long)xi * g.plane + (long long)(row == g.na - 1 ? 0 : row + 1) * g.pb + col;
        const long long ibp = (long long)xi * g.plane + (long long)row * g.pb + (col == g.nb - 1 ? 0 : col + 1);
        for (int q = 0; q < G.neta; ++q) {
            const double* e = eta + (long long)q * g.nstore;
            const double ec = e[idx];
            if (xi < g.nx - 1 || G.x_above) { const double t = (e[ixp] - ec) / G.dx; density += .5 * G.K * (t * t); }
            if (G.dim == 3) {
                { const double t = (e[iap] - ec) / G.da; density += .5 * G.K * (t * t); }
                { const double t = (e[ibp] - ec) / G.db; density += .5 * G.K * (t * t); }
            } else {
                const double t = (e[ibp] - ec) / G.db;
                density += .5 * G.K * (t * t);
            }
        }
        acc[2] = dd_add(acc[2], G.dim == 3 ? density * G.dx * G.da * G.db : density * G.dx * G.db);
    }
    // block reduction
    for (int off = 16; off > 0; off >>= 1) {
        lo = ext_min(lo, shfl_ext(lo, off)); hi = ext_max(hi, shfl_ext(hi, off));
        slo = ext_min(slo, shfl_ext(slo, off)); shi = ext_max(shi, shfl_ext(shi, off));
        gbmax = ext_max(gbmax, shfl_ext(gbmax, off));
    }
    __shared__ Ext se[32][5];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) { se[w][0] = lo; se[w][1] = hi; se[w][2] = slo; se[w][3] = shi; se[w][4] = gbmax; }
    block_reduce<3>(acc, unassigned);
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < nw; ++ww) {
            lo = ext_min(lo, se[ww][0]); hi = ext_max(hi, se[ww][1]);
            slo = ext_min(slo, se[ww][2]); shi = ext_max(shi, se[ww][3]); gbmax = ext_max(gbmax, se[ww][4]);
        }
        GrainPart& o = parts[blockIdx.x];
        for (int q = 0; q < 3; ++q) { o.sum[q][0] = acc[q].hi; o.sum[q][1] = acc[q].lo; }
        o.lo = lo; o.hi = hi; o.slo = slo; o.shi = shi; o.gbmax = gbmax;
        o.unassigned = unassigned;
    }
}

// weighted metal amount of grain q: sum of (1-h) eta_q^2 / S over cells with S > 1e-24
__global__ void k_grain_amount(const GrainParams G, const double* __restrict__ eta, const double* __restrict__ s2,
                               const double* __restrict__ p, double* amount_parts /* [gridDim.x][neta][2] */) {
    const Grid& g = G.g;
    const int q = blockIdx.y;
    DD acc[1] = {{0., 0.}};
    long long dummy = 0;
    const double* e = eta + (long long)q * g.nstore;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const double S = s2[idx];
        if (S > 1.e-24) {
            const double v = e[idx], metal = 1. - h(p[idx]);
            acc[0] = dd_add(acc[0], metal * v * v / S);
        }
    }
    block_reduce<1>(acc, dummy);
    if (threadIdx.x == 0) {
        amount_parts[((long long)blockIdx.x * G.neta + q) * 2] = acc[0].hi;
        amount_parts[((long long)blockIdx.x * G.neta + q) * 2 + 1] = acc[0].lo;
    }
}

__global__ void k_grain_finalize(const GrainParams G, const GrainPart* __restrict__ parts, int nparts,
                                 const double* __restrict__ amount_parts, const unsigned long long* __restrict__ cells,
                                 GrainOut* out, double* amount_out, long long* cells_out) {
    // one thread per grain for the amounts (block order), thread 0 for the scalars
    for (int q = threadIdx.x; q < G.neta; q += blockDim.x) {
        DD a{0., 0.};
        for (int b = 0; b < nparts; ++b)
            a = dd_add(a, DD{amount_parts[((long long)b * G.neta + q) * 2], amount_parts[((long long)b * G.neta + q) * 2 + 1]});
        amount_out[2 * q] = a.hi;
        amount_out[2 * q + 1] = a.lo;
        cells_out[q] = (long long)cells[q];
    }
    if (threadIdx.x == 0) {
        GrainPart r = parts[0];
        for (int b = 1; b < nparts; ++b) {
            for (int q = 0; q < 3; ++q) {
                DD s = dd_add(DD{r.sum[q][0], r.sum[q][1]}, DD{parts[b].sum[q][0], parts[b].sum[q][1]});
                r.sum[q][0] = s.hi; r.sum[q][1] = s.lo;
            }
            r.lo = ext_min(r.lo, parts[b].lo); r.hi = ext_max(r.hi, parts[b].hi);
            r.slo = ext_min(r.slo, parts[b].slo); r.shi = ext_max(r.shi, parts[b].shi);
            r.gbmax = ext_max(r.gbmax, parts[b].gbmax);
            r.unassigned += parts[b].unassigned;
        }
        out->lo = r.lo.v; out->hi = r.hi.v; out->slo = r.slo.v; out->shi = r.shi.v; out->gbmax = r.gbmax.v;
        for (int q = 0; q < 3; ++q) { out->sum[q][0] = r.sum[q][0]; out->sum[q][1] = r.sum[q][1]; }
        out->unassigned = r.unassigned;
    }
}

int grid_for(long long n, int threads, int cap) {
    const long long want = (n + threads - 1) / threads;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

void launch_init_fields(const InitParams& I, double* o, double* cr, double* p, cudaStream_t stream) {
    k_init_fields<<<grid_for(I.g.ncells, 256, 148 * 16), 256, 0, stream>>>(I, o, cr, p);
}
// Seed tables larger than this are read from global memory (200 KB: ~8,500 seeds).
constexpr size_t kSeedSmemMax = 200 * 1024;

void launch_voronoi3(const InitParams& I, const double* seeds, double* grain, double* db, int* volumes,
                     int* competitor, cudaStream_t stream) {
    const size_t sm = (size_t)3 * I.ng * sizeof(double);
    if (sm > kSeedSmemMax) {
        k_voronoi3<false><<<grid_for(I.g.ncells, 128, 148 * 32), 128, 0, stream>>>(I, seeds, grain, db, volumes, competitor);
        return;
    }
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_voronoi3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_voronoi3<true><<<grid_for(I.g.ncells, 128, 148 * 32), 128, sm, stream>>>(I, seeds, grain, db, volumes, competitor);
}
void launch_grain_adjacency(const InitParams& I, const double* grain, unsigned char* adj, cudaStream_t stream) {
    k_grain_adjacency<<<grid_for(I.g.ncells, 256, 148 * 16), 256, 0, stream>>>(I, grain, adj);
}
void launch_eta_dist3(const InitParams& I, const double* seeds, const double* grain, double* eta, cudaStream_t stream) {
    const size_t sm = (size_t)3 * I.ng * sizeof(double);
    if (sm > kSeedSmemMax) {
        k_eta_dist3<false><<<grid_for(I.g.ncells, 128, 148 * 32), 128, 0, stream>>>(I, seeds, grain, eta);
        return;
    }
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_eta_dist3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_eta_dist3<true><<<grid_for(I.g.ncells, 128, 148 * 32), 128, sm, stream>>>(I, seeds, grain, eta);
}
void launch_center_seed(const InitParams& I, double cx, double cy, double cz, double r, int neta, double* o,
                        double* cr, double* p, double* eta, StepPartial* partials, cudaStream_t stream,
                        int* nblocks_out) {
    const int nb = grid_for(I.g.ncells, 256, 148 * 4);
    k_center_seed<<<nb, 256, 0, stream>>>(I, cx, cy, cz, r, neta, o, cr, p, eta, partials);
    *nblocks_out = nb;
}
void launch_reduce_partials(const StepPartial* partials, int nblocks, StepPartial* out, cudaStream_t stream) {
    k_reduce_partials<<<1, 256, 0, stream>>>(partials, nblocks, out);
}
void launch_grain_stats(const GrainParams& G, const double* eta, const double* s2, const double* p, const double* gb,
                        GrainWork& W, GrainOut* out, double* amount_out, long long* cells_out, cudaStream_t stream) {
    const int nb = grid_for(G.g.ncells, 256, 148 * 2);
    cudaMemsetAsync(W.cells, 0, (size_t)G.neta * sizeof(unsigned long long), stream);
    k_grain_scalar<<<nb, 256, 0, stream>>>(G, eta, s2, p, gb, W.cells, reinterpret_cast<GrainPart*>(W.parts));
    k_grain_amount<<<dim3(nb, G.neta), 256, 0, stream>>>(G, eta, s2, p, W.amount_parts);
    k_grain_finalize<<<1, 256, 0, stream>>>(G, reinterpret_cast<const GrainPart*>(W.parts), nb, W.amount_parts, W.cells,
                                           out, amount_out, cells_out);
}
size_t grain_part_bytes() { return sizeof(GrainPart); }
int grain_blocks(long long ncells) { return grid_for(ncells, 256, 148 * 2); }

void launch_diagnostics(const Grid& g, const double* o, const double* cr, const double* p, DiagOut* partials,
                        int* nblocks, DiagOut* out, cudaStream_t stream) {
    const int nb = grid_for(g.ncells, 256, 148 * 4);
    k_diagnostics<<<nb, 256, 0, stream>>>(g, o, cr, p, partials);
    k_diag_finalize<<<1, 32, 0, stream>>>(partials, nb, out);
    if (nblocks) *nblocks = nb;
}

}  // namespace nicr
