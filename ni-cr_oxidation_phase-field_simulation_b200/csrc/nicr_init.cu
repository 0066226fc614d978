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
        if (I.inlet_layer && x == 0) { ov = I.layer_o; cv = Phys::layerCr; }
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

__global__ void k_voronoi3(const InitParams I, const double* __restrict__ seeds, double* grain, double* dbout,
                           int* volumes) {
    extern __shared__ double ss[];
    for (int q = threadIdx.x; q < 3 * I.ng; q += blockDim.x) ss[q] = seeds[q];
    __syncthreads();
    const Grid& g = I.g;
    const int ny = g.na, nz = g.nb;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const double x = (xi + 1) - .5, y = (row + 1) - .5, z = (col + 1) - .5;
        int owner = 0;
        double rbest = CUDART_INF, oY = 0., oZ = 0.;
        for (int s = 0; s < I.ng; ++s) {
            const double yy = min_image(ss[3 * s + 1] - y, I.nyd), zz = min_image(ss[3 * s + 2] - z, I.nzd);
            const double ax = ss[3 * s] - x;
            const double rr = ax * ax + yy * yy + zz * zz;
            if (rr < rbest) { rbest = rr; owner = s; oY = y + yy; oZ = z + zz; }
        }
        double db = CUDART_INF;
        for (int s = 0; s < I.ng; ++s)
            if (s != owner) db = smin(db, competitor_distance(ss, s, owner, x, y, z, oY, oZ, rbest, ny, nz));
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        grain[idx] = owner + 1;
        dbout[idx] = db;
        atomicAdd(volumes + owner, 1);
    }
}

__global__ void k_eta_dist3(const InitParams I, const double* __restrict__ seeds, const double* __restrict__ grain,
                            double* eta) {
    extern __shared__ double ss[];
    for (int q = threadIdx.x; q < 3 * I.ng; q += blockDim.x) ss[q] = seeds[q];
    __syncthreads();
    const Grid& g = I.g;
    const int ny = g.na, nz = g.nb;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncells; c += (long long)gridDim.x * blockDim.x) {
        int xi, row, col;
        decode(g, c, xi, row, col);
        const long long idx = (long long)xi * g.plane + (long long)row * g.pb + col;
        const int owner = (int)grain[idx] - 1;
        const double x = (xi + 1) - .5, y = (row + 1) - .5, z = (col + 1) - .5;
        const double oy = y + min_image(ss[3 * owner + 1] - y, I.nyd), oz = z + min_image(ss[3 * owner + 2] - z, I.nzd);
        const double ax = ss[3 * owner] - x, ay = oy - y, az = oz - z;
        const double rbest = ax * ax + ay * ay + az * az;
        for (int s = 0; s < I.ng; ++s)
            eta[(long long)s * g.nstore + idx] =
                s == owner ? -1. : competitor_distance(ss, s, owner, x, y, z, oy, oz, rbest, ny, nz);
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
        const double ddx = (xi + 1) - cx;
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
            acc[0] = dd_add(acc[0], Phys::oxideO - o[idx]);
            acc[1] = dd_add(acc[1], Phys::oxideCr - cr[idx]);
            o[idx] = Phys::oxideO; cr[idx] = Phys::oxideCr; p[idx] = 1.;
            for (int q = 0; q < neta; ++q) eta[(long long)q * g.nstore + idx] = 0.;
            ++cnt;
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

int grid_for(long long n, int threads, int cap) {
    const long long want = (n + threads - 1) / threads;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

void launch_init_fields(const InitParams& I, double* o, double* cr, double* p, cudaStream_t stream) {
    k_init_fields<<<grid_for(I.g.ncells, 256, 148 * 16), 256, 0, stream>>>(I, o, cr, p);
}
void launch_voronoi3(const InitParams& I, const double* seeds, double* grain, double* db, int* volumes,
                     cudaStream_t stream) {
    const size_t sm = (size_t)3 * I.ng * sizeof(double);
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_voronoi3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_voronoi3<<<grid_for(I.g.ncells, 128, 148 * 32), 128, sm, stream>>>(I, seeds, grain, db, volumes);
}
void launch_eta_dist3(const InitParams& I, const double* seeds, const double* grain, double* eta, cudaStream_t stream) {
    const size_t sm = (size_t)3 * I.ng * sizeof(double);
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_eta_dist3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_eta_dist3<<<grid_for(I.g.ncells, 128, 148 * 32), 128, sm, stream>>>(I, seeds, grain, eta);
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
void launch_diagnostics(const Grid& g, const double* o, const double* cr, const double* p, DiagOut* partials,
                        int* nblocks, DiagOut* out, cudaStream_t stream) {
    const int nb = grid_for(g.ncells, 256, 148 * 4);
    k_diagnostics<<<nb, 256, 0, stream>>>(g, o, cr, p, partials);
    k_diag_finalize<<<1, 32, 0, stream>>>(partials, nb, out);
    if (nblocks) *nblocks = nb;
}

}  // namespace nicr
