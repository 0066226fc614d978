// Convolution kernels of the learned surrogate (a 3D U-Net that proposes the
// state K steps ahead): 3x3x3 convolutions, stride 1, zero padding 1, as
// implicit GEMMs on the BF16 tensor cores with FP32 accumulation.
//
// Layout: activations NDHWC, BF16, channels a multiple of 16; weights
// [Cout][27][Cin] BF16 (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)); outputs FP32.
//   forward  y[v][co]  = sum_{tap,ci} x[v + off(tap)][ci] * w[co][tap][ci]
//            (GEMM: M = voxels, N = Cout, K = 27*Cin; A gathered per tap)
//   dgrad    dx = forward(dy, w') with w'[ci][tap][co] = w[co][26-tap][ci]
//            (off(26 - tap) = -off(tap)); the caller transposes the weights
//   wgrad    dw[co][tap][ci] = sum_v dy[v][co] * x[v + off(tap)][ci]
//            (GEMM per tap: M = Cout, N = Cin, K = voxels, split over CTAs)
// This first form uses the warp-level WMMA tensor-core instructions (16x16x16
// BF16 tiles staged through shared memory with plain 16-byte loads); the
// tcgen05/TMEM form is the next step for these GEMMs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include "../../include/nicr.h"

namespace {

using namespace nvcuda;

struct Vol {
    int n, d, h, w;   // batch and grid
    __host__ __device__ long long voxels() const { return (long long)n * d * h * w; }
};

// voxel index of v shifted by tap, or -1 outside the grid (zero padding)
__device__ __forceinline__ long long shifted(const Vol& V, long long v, int tap) {
    const int x = (int)(v % V.w);
    long long r = v / V.w;
    const int y = (int)(r % V.h);
    r /= V.h;
    const int z = (int)(r % V.d);
    const long long b = r / V.d;
    const int xx = x + tap % 3 - 1, yy = y + (tap / 3) % 3 - 1, zz = z + tap / 9 - 1;
    if (xx < 0 || xx >= V.w || yy < 0 || yy >= V.h || zz < 0 || zz >= V.d) return -1;
    return ((b * V.d + zz) * V.h + yy) * V.w + xx;
}

constexpr int BM = 64, BN = 64, BK = 16;

// Forward: CTA of 4 warps = a 64-voxel x 64-output-channel tile; warp w owns
// voxel rows 16w..16w+15 and the four 16-column accumulators.
__global__ void __launch_bounds__(128) k_conv3d_fwd(const __nv_bfloat16* __restrict__ x,
                                                     const __nv_bfloat16* __restrict__ wt, float* __restrict__ y,
                                                     const Vol V, int cin, int cout) {
    __shared__ __align__(32) __nv_bfloat16 As[BM * BK];   // row-major, ld 16
    __shared__ __align__(32) __nv_bfloat16 Bs[BN * BK];   // col-major (k fastest), ld 16
    const int t = threadIdx.x, warp = t >> 5;
    const long long v0 = (long long)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int ncols = min(BN, cout - n0);
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[4];
    for (int j = 0; j < 4; ++j) wmma::fill_fragment(acc[j], 0.f);
    // thread t stages row t/2 (A: voxel, B: output channel), half t%2 (8 channels)
    const int row = t >> 1, half = t & 1;
    for (int tap = 0; tap < 27; ++tap) {
        const long long src = shifted(V, v0 + row, tap);
        for (int c0 = 0; c0 < cin; c0 += BK) {
            uint4 a = make_uint4(0, 0, 0, 0);
            if (src >= 0) a = *reinterpret_cast<const uint4*>(x + src * cin + c0 + half * 8);
            *reinterpret_cast<uint4*>(As + row * BK + half * 8) = a;
            uint4 b = make_uint4(0, 0, 0, 0);
            if (row < ncols) b = *reinterpret_cast<const uint4*>(wt + ((long long)(n0 + row) * 27 + tap) * cin + c0 + half * 8);
            *reinterpret_cast<uint4*>(Bs + row * BK + half * 8) = b;
            __syncthreads();
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
            wmma::load_matrix_sync(fa, As + warp * 16 * BK, BK);
            for (int j = 0; j < 4; ++j) {
                if (j * 16 >= ncols) break;
                wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> fb;
                wmma::load_matrix_sync(fb, Bs + j * 16 * BK, BK);
                wmma::mma_sync(acc[j], fa, fb, acc[j]);
            }
            __syncthreads();
        }
    }
    for (int j = 0; j < 4; ++j) {
        if (j * 16 >= ncols) break;
        wmma::store_matrix_sync(y + (v0 + warp * 16) * cout + n0 + j * 16, acc[j], cout, wmma::mem_row_major);
    }
}

// Weight gradient: CTA (tap, 16 input channels, 16 output channels, voxel
// slice); 4 warps split the slice, reduce through shared memory, and add the
// 16x16 tile to dw atomically (FP32).
__global__ void __launch_bounds__(128) k_conv3d_wgrad(const __nv_bfloat16* __restrict__ x,
                                                       const __nv_bfloat16* __restrict__ dy, float* __restrict__ dw,
                                                       const Vol V, int cin, int cout, long long slice) {
    __shared__ __align__(32) __nv_bfloat16 Bs[4][16 * 16];   // per warp: 16 voxels x 16 in-channels, row-major
    __shared__ __align__(32) float Cs[4][16 * 16];
    const int tap = blockIdx.x, ci0 = blockIdx.y * 16, co0 = blockIdx.z % (cout / 16) * 16;
    const int part = blockIdx.z / (cout / 16);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const long long M = V.voxels();
    const long long vbeg = (long long)part * slice, vend = min(M, vbeg + slice);
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.f);
    for (long long v = vbeg + warp * 16; v < vend; v += 64) {
        // B: rows = the 16 voxels (shifted by tap, zero outside), cols = 16 in-channels
        {
            const int r = lane >> 1, h = lane & 1;
            const long long s = shifted(V, v + r, tap);
            uint4 b = make_uint4(0, 0, 0, 0);
            if (s >= 0) b = *reinterpret_cast<const uint4*>(x + s * cin + ci0 + h * 8);
            *reinterpret_cast<uint4*>(&Bs[warp][r * 16 + h * 8]) = b;
        }
        __syncwarp();
        // A(co, v) = dy[v][co]: column-major with leading dimension cout
        wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> fa;
        wmma::load_matrix_sync(fa, dy + v * cout + co0, cout);
        wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
        wmma::load_matrix_sync(fb, &Bs[warp][0], 16);
        wmma::mma_sync(acc, fa, fb, acc);
        __syncwarp();
    }
    wmma::store_matrix_sync(&Cs[warp][0], acc, 16, wmma::mem_row_major);
    __syncthreads();
    for (int q = t; q < 256; q += 128) {
        const float s = Cs[0][q] + Cs[1][q] + Cs[2][q] + Cs[3][q];
        const int co = q / 16, ci = q % 16;
        atomicAdd(dw + ((long long)(co0 + co) * 27 + tap) * cin + ci0 + ci, s);
    }
}

int check_args(long long voxels, int cin, int cout) {
    if (voxels <= 0 || voxels % 64 != 0 || cin <= 0 || cin % 16 != 0 || cout <= 0 || cout % 16 != 0)
        return NICR_ERR_INVALID_ARG;
    return NICR_OK;
}

}  // namespace

extern "C" {

int nicr_conv3d_fwd(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                    void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !w || !y) return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const dim3 grid((unsigned)(V.voxels() / BM), (unsigned)((cout + BN - 1) / BN));
    k_conv3d_fwd<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), y, V, cin, cout);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

int nicr_conv3d_wgrad(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                      void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !dy || !dw) return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long M = V.voxels();
    // enough voxel slices to fill the GPU: 27 x (Cin/16) x (Cout/16) x parts CTAs
    const long long tiles = 27LL * (cin / 16) * (cout / 16);
    long long parts = (148LL * 8 + tiles - 1) / tiles;
    long long slice = (M + parts - 1) / parts;
    slice = (slice + 63) / 64 * 64;
    parts = (M + slice - 1) / slice;
    cudaMemsetAsync(dw, 0, sizeof(float) * (size_t)cout * 27 * cin, s);
    const dim3 grid(27, (unsigned)(cin / 16), (unsigned)((cout / 16) * parts));
    k_conv3d_wgrad<<<grid, 128, 0, s>>>(static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw,
                                        V, cin, cout, slice);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

}  // extern "C"
