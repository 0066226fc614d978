// Convolution kernels of the learned surrogate (a 3D U-Net that proposes the
// state K steps ahead): 3x3x3 convolutions, stride 1, zero padding 1, as
// implicit GEMMs on the BF16 tensor cores with FP32 accumulation.
//
// Layout: activations NDHWC, BF16, channels a multiple of 16; weights
// [Cout][27][Cin] BF16 (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)); outputs FP32
// (or, through the fused epilogue, act(y + bias) in BF16).
//   forward  y[v][co]  = sum_{tap,ci} x[v + off(tap)][ci] * w[co][tap][ci]
//            (GEMM: M = voxels, N = Cout, K = 27*Cin)
//   dgrad    dx = forward(dy, w') with w'[ci][tap][co] = w[co][26-tap][ci]
//            (off(26 - tap) = -off(tap)); the caller transposes the weights
//   wgrad    dw[co][tap][ci] = sum_v dy[v][co] * x[v + off(tap)][ci]
//            (GEMM: M = (tap, Cout), N = Cin, K = voxels, split over CTAs)
// Every tcgen05 form keeps its accumulator in TMEM. Forward forms, chosen by
// shape in nicr_conv3d_fwd_act from measured rates:
//   k_conv3d_fwd_march  Cin 16, rows >= 128: halo lines kept on chip along y
//   k_conv3d_fwd_halo   narrow outputs, rows >= 128: one halo block per chunk
//   k_conv3d_fwd_tma    everything else: per-tap TMA boxes
//   k_conv3d_fwd_tc     where the driver refuses a tensor map: cp.async gathers
// The weight gradient runs on tcgen05.mma with TMA-staged operands
// (k_conv3d_wgrad_tma) for Cout 16, 32, 64 or multiples of 128. The
// warp-level WMMA forms (16x16x16 BF16 tiles staged through shared memory)
// stay as reference forms and as the weight gradient of other Cout.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <mma.h>

#include <map>
#include <mutex>
#include <utility>

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

// ---------------------------------------------------------------- tcgen05
// Forward on the 5th-generation tensor cores: CTA of 4 warps = 128 voxels x
// N output channels (N <= 256), accumulator in TMEM (128 lanes x N FP32
// columns). The K loop runs over 27 taps x Cin/KC chunks; each chunk (stage)
// is gathered by all threads with zero-filling 16-byte cp.async into the
// no-swizzle K-major canonical layout (8-row x 16-byte core matrices; chunk
// (row r, 16-byte column kc) at byte kc*ROWS*16 + r*16, so SBO = 128 B between
// 8-row groups and LBO = ROWS*16 B between the two K halves of an MMA), and
// one thread issues its KC/16 tcgen05.mma (M=128, N, K=16; BF16 in, FP32
// accumulate) and commits them to the stage's mbarrier. Four stages, loads
// run two chunks ahead. Every mbarrier wait is bounded: on timeout the CTA
// records the error, stops issuing work, waits (bounded) for its MMAs and
// frees its TMEM.
constexpr int TC_M = 128, TC_STAGES = 4, TC_AHEAD = 2;
constexpr long long TC_SPIN = 1LL << 22;

__device__ int g_conv_error;   // non-zero after a timed-out wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);   // version 1, no swizzle
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < TC_SPIN; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(128) k_conv3d_fwd_tc(const __nv_bfloat16* __restrict__ x,
                                                        const __nv_bfloat16* __restrict__ wt, float* __restrict__ y,
                                                        const Vol V, int cin, int cout, int kc_elems, int tmem_cols) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const long long M = V.voxels();
    const long long v0 = (long long)blockIdx.x * TC_M;
    const int n0 = blockIdx.y * 256;
    const int N = min(256, cout - n0);
    const int kcols = kc_elems / 8;                      // 16-byte columns per chunk
    const uint32_t a_bytes = TC_M * kc_elems * 2, b_bytes = (uint32_t)N * kc_elems * 2;
    const uint32_t stage_bytes = (a_bytes + b_bytes + 1023) & ~1023u;
    unsigned char* stages = tc_smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + TC_STAGES * stage_bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + TC_STAGES);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        for (int s = 0; s < TC_STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int chunks_per_tap = cin / kc_elems;
    const int iters = 27 * chunks_per_tap;
    const uint32_t idesc = umma_idesc(TC_M, N);
    const bool row_ok = v0 + t < M;

    auto load = [&](int it) {
        const int tap = it / chunks_per_tap, c0 = (it % chunks_per_tap) * kc_elems;
        const uint32_t base = smem_u32(stages + (it % TC_STAGES) * stage_bytes);
        const long long src = row_ok ? shifted(V, v0 + t, tap) : -1;
        const __nv_bfloat16* a_src = src >= 0 ? x + src * cin + c0 : x;
        for (int kc = 0; kc < kcols; ++kc)   // A: thread t owns voxel row t
            cp_async16(base + (uint32_t)(kc * TC_M + t) * 16, a_src + (src >= 0 ? kc * 8 : 0), src >= 0);
        for (int q = t; q < kcols * N; q += 128) {   // B: chunk q = kc * N + co
            const int kc = q / N, co = q % N;
            cp_async16(base + a_bytes + (uint32_t)q * 16, wt + ((long long)(n0 + co) * 27 + tap) * cin + c0 + kc * 8, true);
        }
    };

    for (int it = 0; it < TC_AHEAD && it < iters; ++it) {
        load(it);
        asm volatile("cp.async.commit_group;");
    }
    bool ok = true;
    int committed = 0;   // chunks whose MMAs have been issued and committed
    for (int it = 0; it < iters; ++it) {
        const int ahead = it + TC_AHEAD;
        if (ahead < iters) {
            // the stage of chunk `ahead` last held chunk ahead - STAGES: its MMAs must have finished
            if (ahead >= TC_STAGES)
                ok = mbar_wait(smem_u32(bars + ahead % TC_STAGES), (uint32_t)((ahead / TC_STAGES - 1) & 1));
            if (__syncthreads_or(!ok)) break;
            load(ahead);
        }
        asm volatile("cp.async.commit_group;");
        asm volatile("cp.async.wait_group %0;" ::"n"(TC_AHEAD));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = smem_u32(stages + (it % TC_STAGES) * stage_bytes);
            for (int k = 0; k < kc_elems / 16; ++k) {
                const uint64_t ad = umma_sdesc(base + k * 2 * TC_M * 16, TC_M * 16, 128);
                const uint64_t bd = umma_sdesc(base + a_bytes + k * 2 * N * 16, N * 16, 128);
                const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(bars + it % TC_STAGES)));
        }
        committed = it + 1;
    }
    asm volatile("cp.async.wait_all;");
    // the last commit covers every MMA issued before it (also after a timeout,
    // so that no MMA is in flight when the TMEM is freed)
    if (committed > 0) {
        const int last = committed - 1;
        const bool done = mbar_wait(smem_u32(bars + last % TC_STAGES), (uint32_t)((last / TC_STAGES) & 1));
        ok = ok && done;
    }
    ok = !__syncthreads_or(!ok);
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const bool store = v0 + warp * 32 + lane < M;
        float* out = y + (v0 + warp * 32 + lane) * cout + n0;
        for (int c = 0; c < N; c += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (store)
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(out + c + j) =
                        make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                                    __uint_as_float(r[j + 3]));
        }
    } else if (t == 0) {
        atomicExch(&g_conv_error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ---------------------------------------------------------------- tcgen05 + TMA
// The forward with both operands staged by the tensor memory accelerator.
// Output tile: Wt x Ht voxels of one (batch, z) plane (Wt * Ht = 128 rows of
// the MMA) x N output channels. Per chunk (tap, KC channels):
//   A = the 5D box {KC, Wt, Ht, 1, 1} of x at (c0, x0+dx, y0+dy, z+dz, b):
//       out-of-range coordinates read zeros, which is the convolution's zero
//       padding, so every tap is a plain coordinate offset;
//   B = the 3D box {KC, 1, N} of w at (c0, tap, n0).
// Both land K-major with the swizzle matching KC (64 -> 128 B, 32 -> 64 B,
// 16 -> 32 B rows), the canonical layouts tcgen05.mma reads (8-row groups
// SBO = 8 rows apart; K steps of 16 advance the start address by 32 B).
// Warp 0 lane 0 issues the loads (full barrier: expect_tx), warp 1 lane 0
// the MMAs (stage freed through its empty barrier by tcgen05.commit), all
// four warps the epilogue. Waits are bounded as in k_conv3d_fwd_tc.
struct TmaConv {
    int kc, swz_bytes, stages, wt, ht, tiles_x, tiles_y, cols;
    uint32_t a_bytes, b_bytes, stage_bytes;
    size_t smem;
};

__device__ __forceinline__ uint64_t umma_sdesc_sw(uint32_t saddr, uint32_t row_bytes) {
    const uint64_t layout = row_bytes == 128 ? 2 : row_bytes == 64 ? 4 : 6;   // SWIZZLE_128B / 64B / 32B
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) |                 // LBO unused (1)
           ((uint64_t)(((8 * row_bytes) >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (layout << 61);
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                       uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
        "[%7];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// Epilogue options of the TMA forward (act): bias added per output channel
// when `bias` is given, then ACT_RELU, and the result stored as BF16 with
// ACT_BF16 (else FP32).
constexpr int ACT_RELU = 1, ACT_BF16 = 2;

__global__ void __launch_bounds__(128) k_conv3d_fwd_tma(const __grid_constant__ CUtensorMap xmap,
                                                         const __grid_constant__ CUtensorMap wmap, void* __restrict__ y,
                                                         const float* __restrict__ bias, int act, const Vol V, int cin,
                                                         int cout, const TmaConv C) {
    extern __shared__ unsigned char tma_smem_raw[];
    const uint32_t raw = smem_u32(tma_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;   // swizzled stages start on 1024-byte boundaries
    unsigned char* gen = tma_smem_raw + (base - raw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int S = C.stages;
    uint64_t* full = reinterpret_cast<uint64_t*>(gen + S * C.stage_bytes);
    uint64_t* empty = full + S;
    uint64_t* acc_full = empty + S;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);
    int* failed = reinterpret_cast<int*>(tmem_slot + 1);
    int* issued = failed + 1;     // chunks whose loads were issued
    int* consumed = failed + 2;   // chunks whose loads the MMA thread saw land

    long long tile = blockIdx.x;
    const int tx = (int)(tile % C.tiles_x);
    tile /= C.tiles_x;
    const int ty = (int)(tile % C.tiles_y);
    tile /= C.tiles_y;
    const int z = (int)(tile % V.d);
    const int b = (int)(tile / V.d);
    const int x0 = tx * C.wt, y0 = ty * C.ht;
    const int n0 = blockIdx.y * 256;
    const int N = min(256, cout - n0);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(C.cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 32) {
        for (int s = 0; s < 2 * S + 1; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        *failed = *issued = *consumed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int chunks_per_tap = cin / C.kc;
    const int iters = 27 * chunks_per_tap;
    if (t == 0) {   // producer
        asm volatile("prefetch.tensormap [%0];" ::"l"(&xmap) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&wmap) : "memory");
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            if (it >= S && !mbar_wait(smem_u32(empty + s), (uint32_t)((it / S - 1) & 1))) {
                atomicExch(failed, 1);
                break;
            }
            const int tap = it / chunks_per_tap, c0 = (it % chunks_per_tap) * C.kc;
            const uint32_t st = base + s * C.stage_bytes;
            // the boxes' full bytes arrive, zero-filled parts included
            mbar_expect(smem_u32(full + s), C.a_bytes + C.b_bytes);
            tma_5d(st, &xmap, c0, x0 + tap % 3 - 1, y0 + (tap / 3) % 3 - 1, z + tap / 9 - 1, b, smem_u32(full + s));
            tma_3d(st + C.a_bytes, &wmap, c0, tap, n0, smem_u32(full + s));
            *issued = it + 1;
        }
    } else if (t == 32) {   // MMA issuer
        const uint32_t idesc = umma_idesc(TC_M, N);
        const uint32_t row = (uint32_t)C.swz_bytes;
        int it = 0;
        for (; it < iters; ++it) {
            const int s = it % S;
            if (!mbar_wait(smem_u32(full + s), (uint32_t)((it / S) & 1))) {
                atomicExch(failed, 1);
                break;
            }
            *consumed = it + 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + s * C.stage_bytes;
            for (int k = 0; k < C.kc / 16; ++k) {
                const uint64_t ad = umma_sdesc_sw(st + k * 32, row);
                const uint64_t bd = umma_sdesc_sw(st + C.a_bytes + k * 32, row);
                const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(empty + s)));
        }
        // arrives once every MMA issued so far has completed (also after a timeout)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(acc_full)));
    }
    __syncwarp();
    bool ok = mbar_wait(smem_u32(acc_full), 0);
    __syncthreads();
    ok = ok && *failed == 0;
    if (!__syncthreads_or(!ok)) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = warp * 32 + lane;
        const int yy = y0 + r / C.wt, xx = x0 + r % C.wt;
        const bool store = yy < V.h && xx < V.w;
        const long long o0 = ((((long long)b * V.d + z) * V.h + yy) * V.w + xx) * cout + n0;
        for (int c = 0; c < N; c += 16) {
            uint32_t q[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
                  "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j += 4) {
                const float4 bj = bias ? *reinterpret_cast<const float4*>(bias + n0 + c + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                v[j] = __uint_as_float(q[j]) + bj.x;
                v[j + 1] = __uint_as_float(q[j + 1]) + bj.y;
                v[j + 2] = __uint_as_float(q[j + 2]) + bj.z;
                v[j + 3] = __uint_as_float(q[j + 3]) + bj.w;
            }
            if (act & ACT_RELU) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.f);
            }
            if (!store) continue;
            if (act & ACT_BF16) {
                uint32_t h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    h[j] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * j])) |
                           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * j + 1])) << 16);
                uint4* out = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + o0 + c);
                out[0] = make_uint4(h[0], h[1], h[2], h[3]);
                out[1] = make_uint4(h[4], h[5], h[6], h[7]);
            } else {
                float* out = static_cast<float*>(y) + o0 + c;
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(out + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            }
        }
    } else if (t == 0) {
        atomicExch(&g_conv_error, 1);
        // loads still in flight land in this CTA's shared memory: wait (bounded) for the issued ones
        for (int it = *consumed; it < *issued; ++it) mbar_wait(smem_u32(full + it % S), (uint32_t)((it / S) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C.cols));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the CUDA runtime statically and not libcuda).
PFN_cuTensorMapEncodeTiled_v12000 conv_map_encoder() {
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

TmaConv tma_conv_plan(const Vol& V, int cin, int cout) {
    TmaConv C{};
    C.kc = cin % 64 == 0 ? 64 : cin % 32 == 0 ? 32 : 16;
    C.swz_bytes = C.kc * 2;
    C.wt = 1;
    while (C.wt < V.w && C.wt < TC_M) C.wt <<= 1;
    C.ht = TC_M / C.wt;
    C.tiles_x = (V.w + C.wt - 1) / C.wt;
    C.tiles_y = (V.h + C.ht - 1) / C.ht;
    const int cmax = cout < 256 ? cout : 256;
    C.cols = 32;
    while (C.cols < cmax) C.cols <<= 1;
    C.a_bytes = (uint32_t)TC_M * C.kc * 2;
    C.b_bytes = (uint32_t)cmax * C.kc * 2;
    C.stage_bytes = (C.a_bytes + C.b_bytes + 1023u) & ~1023u;
    // about 72 KB of stages (at least 2): two or three CTAs share an SM, so one
    // CTA's epilogue overlaps another's main loop (64->256 at 64^3: 1029
    // TFLOP/s, against 808 with 200 KB and one CTA per SM)
    C.stages = (int)((72u * 1024u) / C.stage_bytes);
    if (C.stages < 2) C.stages = 2;
    if (C.stages > 8) C.stages = 8;
    // barriers (2 per stage + 1), the TMEM address and the failure flag, and
    // 1 KB to align the stages; at least cols x 400 bytes (TMEM per SM)
    C.smem = (size_t)C.stages * C.stage_bytes + (2 * C.stages + 1) * 8 + 16 + 1024;
    if (C.smem < (size_t)C.cols * 400) C.smem = (size_t)C.cols * 400;
    return C;
}

// ---------------------------------------------------------------- forward from a halo block
// For narrow outputs (Cout <= 64) on rows of at least 128 voxels: the
// output tile is 128 consecutive voxels of one x row (b, z, y, x0..x0+127).
// Per chunk of 16 input channels, two TMA boxes {8, 130, 3, 3, 1} of x at
// (c0 + 8 kc, x0 - 1, y - 1, z - 1, b) bring the whole 3 x 3 x 130 halo block
// into shared memory in the no-swizzle K-major layout, one plane per 8
// channels: row (line, xr) at byte (line * 130 + xr) * 16, line = (dz+1)*3 +
// (dy+1). The A operand of tap (dz, dy, dx) is then the 128 rows starting at
// line * 130 + dx + 1: a descriptor whose start address moves by 16 bytes per
// row (SBO 128 B between 8-row groups, LBO = one plane between the two K
// halves), so x is staged once per chunk instead of once per tap. The
// chunk's weights for all 27 taps are copied by all threads into
// [tap][kc][co][16 B] (LBO = Cout * 16 B). Zero fill outside the grid is the
// padding. Stages: one per chunk in flight (two when Cin > 16).
constexpr int HB_ROWS = 130, HB_LINES = 9;

struct HaloConv {
    int chunks, stages, cols, tiles_x;
    uint32_t a_box, a_plane, a_bytes, b_bytes, stage_bytes;   // a_plane: a_box rounded up to 128 bytes
    size_t smem;
};

__global__ void __launch_bounds__(128) k_conv3d_fwd_halo(const __grid_constant__ CUtensorMap xmap,
                                                          const __nv_bfloat16* __restrict__ wt, void* __restrict__ y,
                                                          const float* __restrict__ bias, int act, const Vol V, int cin,
                                                          int cout, const HaloConv H) {
    extern __shared__ unsigned char hb_smem_raw[];
    const uint32_t raw = smem_u32(hb_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gen = hb_smem_raw + (base - raw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int S = H.stages;
    uint64_t* full = reinterpret_cast<uint64_t*>(gen + S * H.stage_bytes);
    uint64_t* empty = full + S;
    uint64_t* acc_full = empty + S;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);

    long long tile = blockIdx.x;
    const int tx = (int)(tile % H.tiles_x);
    tile /= H.tiles_x;
    const int yv = (int)(tile % V.h);
    tile /= V.h;
    const int z = (int)(tile % V.d), b = (int)(tile / V.d);
    const int x0 = tx * TC_M;
    const int N = cout;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(H.cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        for (int s = 0; s < 2 * S + 1; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&xmap) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc(TC_M, N);

    bool ok = true;
    int committed = 0;
    for (int c = 0; c < H.chunks; ++c) {
        const int s = c % S;
        const uint32_t st = base + s * H.stage_bytes;
        // the stage last held chunk c - S: its MMAs must have finished
        if (c >= S) ok = mbar_wait(smem_u32(empty + s), (uint32_t)((c / S - 1) & 1));
        if (__syncthreads_or(!ok)) break;
        if (t == 0) {
            mbar_expect(smem_u32(full + s), 2 * H.a_box);
            for (int kc = 0; kc < 2; ++kc)
                tma_5d(st + kc * H.a_plane, &xmap, c * 16 + kc * 8, x0 - 1, yv - 1, z - 1, b, smem_u32(full + s));
        }
        // weights of the chunk: [tap][kc][co][8 channels]
        for (int q = t; q < 27 * 2 * N; q += 128) {
            const int co = q % N, kc = (q / N) % 2, tap = q / (2 * N);
            cp_async16(st + H.a_bytes + (uint32_t)q * 16, wt + ((long long)co * 27 + tap) * cin + c * 16 + kc * 8, true);
        }
        asm volatile("cp.async.commit_group;");
        asm volatile("cp.async.wait_group 0;");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            ok = mbar_wait(smem_u32(full + s), (uint32_t)((c / S) & 1));
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int tap = 0; tap < 27; ++tap) {
                    const uint32_t row = (uint32_t)((tap / 3) * HB_ROWS + tap % 3);
                    const uint64_t ad = umma_sdesc(st + row * 16, H.a_plane, 128);
                    const uint64_t bd = umma_sdesc(st + H.a_bytes + (uint32_t)(tap * 2 * N) * 16, (uint32_t)N * 16, 128);
                    const uint32_t accum = (c > 0 || tap > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(accum));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(empty + s)));
            }
        }
        if (__syncthreads_or(!ok)) break;
        committed = c + 1;
    }
    if (t == 0) asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(acc_full)));
    if (committed > 0 || !ok) {
        const bool done = mbar_wait(smem_u32(acc_full), 0);
        ok = ok && done;
    }
    ok = !__syncthreads_or(!ok);
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = warp * 32 + lane;
        const int xx = x0 + r;
        const bool store = xx < V.w;
        const long long o0 = ((((long long)b * V.d + z) * V.h + yv) * V.w + xx) * cout;
        for (int c = 0; c < N; c += 16) {
            uint32_t q[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
                  "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j += 4) {
                const float4 bj = bias ? *reinterpret_cast<const float4*>(bias + c + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                v[j] = __uint_as_float(q[j]) + bj.x;
                v[j + 1] = __uint_as_float(q[j + 1]) + bj.y;
                v[j + 2] = __uint_as_float(q[j + 2]) + bj.z;
                v[j + 3] = __uint_as_float(q[j + 3]) + bj.w;
            }
            if (act & ACT_RELU) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.f);
            }
            if (!store) continue;
            if (act & ACT_BF16) {
                uint32_t hh[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    hh[j] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * j])) |
                            ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * j + 1])) << 16);
                uint4* out = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + o0 + c);
                out[0] = make_uint4(hh[0], hh[1], hh[2], hh[3]);
                out[1] = make_uint4(hh[4], hh[5], hh[6], hh[7]);
            } else {
                float* out = static_cast<float*>(y) + o0 + c;
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4*>(out + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            }
        }
    } else if (t == 0) {
        atomicExch(&g_conv_error, 1);
        // a chunk's loads may still be in flight: wait (bounded) for the last issued one
        if (committed < H.chunks) mbar_wait(smem_u32(full + committed % S), (uint32_t)((committed / S) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(H.cols));
}

// The halo-block plan, or false outside its shapes (Cout <= 64, W >= 128).
bool halo_plan(const Vol& V, int cin, int cout, HaloConv& H) {
    if (cout > 64 || V.w < TC_M || cin % 16 != 0) return false;
    H = HaloConv{};
    H.chunks = cin / 16;
    H.stages = H.chunks > 1 ? 2 : 1;
    H.cols = 32;
    while (H.cols < cout) H.cols <<= 1;
    H.tiles_x = (V.w + TC_M - 1) / TC_M;
    H.a_box = (uint32_t)HB_LINES * HB_ROWS * 16;
    H.a_plane = (H.a_box + 127u) & ~127u;
    H.a_bytes = 2 * H.a_plane;
    H.b_bytes = (uint32_t)27 * 2 * cout * 16;
    H.stage_bytes = (H.a_bytes + H.b_bytes + 1023u) & ~1023u;
    H.smem = (size_t)H.stages * H.stage_bytes + (2 * H.stages + 1) * 8 + 8 + 1024;
    if (H.smem < (size_t)H.cols * 400) H.smem = (size_t)H.cols * 400;
    return true;
}

// ---------------------------------------------------------------- forward marching along y
// The halo-block forward with the block kept between output lines: a CTA
// owns x tile x0..x0+127 of plane (b, z) and output lines y0..y1-1. Input
// line L (y index; the three z lines z-1..z+1 of it) sits in ring slot L % 4
// as one TMA box {8, 130, 1, 3, 1} per 8 channels ([slot][kc][dz][130 rows]
// [16 B], each box padded to 128 bytes), so a new output line loads 3 input
// lines instead of 9. All weights ([chunk][tap][kc][co][16 B]) are staged
// once per CTA. Two TMEM accumulators: in iteration y the MMAs of line y run
// while the four warps store line y-1; then line y+2 is loaded into the slot
// of line y-2, whose last reader (the MMAs of line y-1) has finished.
// Applies to Cin <= 48, Cout <= 32 on rows of at least 128 voxels.
struct MarchConv {
    int kcp, cols, tiles_x, ysplit, lines;   // 8-channel planes, TMEM columns, x tiles, y ranges, lines per CTA
    uint32_t box, plane, slot, w_bytes, w_off;
    size_t smem;
};

__global__ void __launch_bounds__(128) k_conv3d_fwd_march(const __grid_constant__ CUtensorMap xmap,
                                                           const __nv_bfloat16* __restrict__ wt, void* __restrict__ y,
                                                           const float* __restrict__ bias, int act, const Vol V, int cin,
                                                           int cout, const MarchConv M) {
    extern __shared__ unsigned char mc_smem_raw[];
    const uint32_t raw = smem_u32(mc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gen = mc_smem_raw + (base - raw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    uint64_t* full = reinterpret_cast<uint64_t*>(gen + M.w_off + M.w_bytes);   // 4 slots
    uint64_t* accf = full + 4;                                                 // 2 accumulators
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 2);

    long long blk = blockIdx.x;
    const int tx = (int)(blk % M.tiles_x);
    blk /= M.tiles_x;
    const int ys = (int)(blk % M.ysplit);
    blk /= M.ysplit;
    const int z = (int)(blk % V.d), b = (int)(blk / V.d);
    const int x0 = tx * TC_M, N = cout;
    const int y0 = ys * M.lines, y1 = min(V.h, y0 + M.lines);
    const int chunks = cin / 16;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(M.cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // input line L into its slot (thread 0); k = L - (y0 - 1) counts the loads of this CTA
    auto load_line = [&](int L) {
        const uint32_t sl = (uint32_t)(L - (y0 - 1)) % 4u;
        mbar_expect(smem_u32(full + sl), (uint32_t)M.kcp * M.box);
        for (int kc = 0; kc < M.kcp; ++kc)
            tma_5d(base + sl * M.slot + kc * M.plane, &xmap, kc * 8, x0 - 1, L, z - 1, b, smem_u32(full + sl));
    };
    if (t == 0) {
        for (int s = 0; s < 6; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&xmap) : "memory");
        for (int L = y0 - 1; L <= y0 + 1; ++L) load_line(L);
    }
    // all weights: [chunk][tap][kc][co][8 channels]
    for (int q = t; q < chunks * 27 * 2 * N; q += 128) {
        const int co = q % N, kc = (q / N) % 2, tap = (q / (2 * N)) % 27, c = q / (54 * N);
        cp_async16(base + M.w_off + (uint32_t)q * 16, wt + ((long long)co * 27 + tap) * cin + c * 16 + kc * 8, true);
    }
    asm volatile("cp.async.commit_group;");
    asm volatile("cp.async.wait_group 0;");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc(TC_M, N);

    // stores output line yo from accumulator j % 2 (j = yo - y0) after its MMAs completed
    auto epilogue = [&](int yo) -> bool {
        const int j = yo - y0;
        const bool done = mbar_wait(smem_u32(accf + (j & 1)), (uint32_t)((j >> 1) & 1));
        if (__syncthreads_or(!done)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = warp * 32 + lane;
        const int xx = x0 + r;
        const bool store = xx < V.w;
        const long long o0 = ((((long long)b * V.d + z) * V.h + yo) * V.w + xx) * cout;
        for (int c = 0; c < N; c += 16) {
            uint32_t q[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((j & 1) * N + c);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
                  "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int jj = 0; jj < 16; jj += 4) {
                const float4 bj = bias ? *reinterpret_cast<const float4*>(bias + c + jj) : make_float4(0.f, 0.f, 0.f, 0.f);
                v[jj] = __uint_as_float(q[jj]) + bj.x;
                v[jj + 1] = __uint_as_float(q[jj + 1]) + bj.y;
                v[jj + 2] = __uint_as_float(q[jj + 2]) + bj.z;
                v[jj + 3] = __uint_as_float(q[jj + 3]) + bj.w;
            }
            if (act & ACT_RELU) {
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) v[jj] = fmaxf(v[jj], 0.f);
            }
            if (!store) continue;
            if (act & ACT_BF16) {
                uint32_t hh[8];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj)
                    hh[jj] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * jj])) |
                             ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * jj + 1])) << 16);
                uint4* out = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + o0 + c);
                out[0] = make_uint4(hh[0], hh[1], hh[2], hh[3]);
                out[1] = make_uint4(hh[4], hh[5], hh[6], hh[7]);
            } else {
                float* out = static_cast<float*>(y) + o0 + c;
#pragma unroll
                for (int jj = 0; jj < 16; jj += 4)
                    *reinterpret_cast<float4*>(out + jj) = make_float4(v[jj], v[jj + 1], v[jj + 2], v[jj + 3]);
            }
        }
        // the accumulator is read: the MMAs of line yo + 2 may overwrite it
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        return true;
    };

    bool ok = true;
    int issued = 0;   // output lines whose MMAs were issued
    for (int yo = y0; yo < y1 && ok; ++yo) {
        if (t == 0) {
            // lines yo-1 and yo landed in earlier iterations (or the prologue); wait for yo + 1
            for (int L = (yo == y0 ? yo - 1 : yo + 1); L <= yo + 1 && ok; ++L) {
                const int k = L - (y0 - 1);
                ok = mbar_wait(smem_u32(full + (k & 3)), (uint32_t)((k >> 2) & 1));
            }
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int j = yo - y0;
                const uint32_t dacc = tmem + (uint32_t)((j & 1) * N);
                int first = 1;
                for (int c = 0; c < chunks; ++c)
                    for (int tap = 0; tap < 27; ++tap) {
                        const int L = yo + (tap / 3) % 3 - 1, dz = tap / 9;   // input line and its z line
                        const uint32_t sl = (uint32_t)(L - (y0 - 1)) % 4u;
                        const uint32_t a = base + sl * M.slot + (uint32_t)(2 * c) * M.plane +
                                           (uint32_t)(dz * HB_ROWS + tap % 3) * 16;
                        const uint64_t ad = umma_sdesc(a, M.plane, 128);
                        const uint64_t bd =
                            umma_sdesc(base + M.w_off + (uint32_t)((c * 27 + tap) * 2 * N) * 16, (uint32_t)N * 16, 128);
                        const uint32_t accum = first ? 0u : 1u;
                        first = 0;
                        asm volatile(
                            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dacc),
                            "l"(ad), "l"(bd), "r"(idesc), "r"(accum));
                    }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(accf + (j & 1))));
            }
        }
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        issued = yo - y0 + 1;
        // line yo - 1 out while the MMAs of line yo run
        if (yo > y0 && !epilogue(yo - 1)) {
            ok = false;
            break;
        }
        // the MMAs of line yo - 1 are complete: line yo - 2's slot takes line yo + 2
        if (t == 0 && yo + 2 <= y1) load_line(yo + 2);
    }
    if (ok && issued > 0) ok = epilogue(y0 + issued - 1);
    if (!ok && t == 0) {
        atomicExch(&g_conv_error, 1);
        // wait (bounded) for the issued MMAs and the loads in flight
        if (issued > 0) mbar_wait(smem_u32(accf + ((issued - 1) & 1)), (uint32_t)(((issued - 1) >> 1) & 1));
        const int last = min(y1, y0 + issued + 1);
        for (int L = max(y0 - 1, last - 3); L <= last; ++L) {
            const int k = L - (y0 - 1);
            mbar_wait(smem_u32(full + (k & 3)), (uint32_t)((k >> 2) & 1));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(M.cols));
}

// The y-march plan, or false outside its shapes.
bool march_plan(const Vol& V, int cin, int cout, MarchConv& M) {
    if (cout > 32 || cin > 48 || V.w < TC_M || cin % 16 != 0) return false;
    M = MarchConv{};
    M.kcp = cin / 8;
    M.cols = 32;
    while (M.cols < 2 * cout) M.cols <<= 1;
    M.tiles_x = (V.w + TC_M - 1) / TC_M;
    M.box = 3u * HB_ROWS * 16;
    M.plane = (M.box + 127u) & ~127u;
    M.slot = (uint32_t)M.kcp * M.plane;
    M.w_off = 4 * M.slot;
    M.w_bytes = (uint32_t)27 * cin * cout * 2;
    // y ranges: about 12 CTAs per SM (4 waves at 3 resident), at least 8 lines
    // each; 16->16 at 128^3 (BF16 out): 233 TFLOP/s, against 199 with 4 per SM
    const long long planes = (long long)M.tiles_x * V.d * V.n;
    long long split = (148LL * 12 + planes - 1) / planes;
    if (split > (V.h + 7) / 8) split = (V.h + 7) / 8;
    if (split < 1) split = 1;
    M.lines = (int)((V.h + split - 1) / split);
    M.ysplit = (V.h + M.lines - 1) / M.lines;
    M.smem = (size_t)M.w_off + M.w_bytes + 6 * 8 + 8 + 1024;
    if (M.smem < (size_t)M.cols * 400) M.smem = (size_t)M.cols * 400;
    return M.smem <= 227u * 1024u;
}

// ---------------------------------------------------------------- weight gradient, tcgen05 + TMA
// dw[co][tap][ci] = sum_u dy[u - off(tap)][co] * x[u][ci] (u runs over the
// voxels of x; dy is zero outside the grid): one GEMM with M = (tap, co)
// rows, N = ci, K = voxels. An M tile holds 128/Cout taps of all Cout
// channels (Cout 16, 32 or 64) or 128 channels of one tap (Cout a multiple of
// 128); K advances by tiles of kt voxels (Wt x Ht of one (batch, z) plane) and
// is split over CTAs, which add their partial sums to dw with FP32 atomics.
// Per K tile: A = for each tap of the M tile, the box {Ws_a, Wt, Ht, 1, 1} of
// dy at (co0, x0-dx, y0-dy, z-dz, b) (zero fill = zero outside); B = the
// boxes {Ws_b, Wt, Ht, 1, 1} of x at (ci0, x0, y0, z, b). Both land MN-major
// (rows = the kt voxels, each row Ws channels), with the swizzle of Ws
// (64 -> 128 B, 32 -> 64 B, 16 -> 32 B): 8-row groups SBO = 8 rows apart, the
// blocks of Ws channels LBO = one box apart; an MMA (K = 16) takes two
// 8-row groups.
struct TmaWgrad {
    int kt, wsa, wsb, taps_per_m, m_tiles, co_blocks, n_tiles, wt, ht, tiles_x, tiles_y, ktiles, parts, per_part,
        stages, cols;
    uint32_t a_box, b_box, a_bytes, b_bytes, stage_bytes;
    size_t smem;
};

// voxels per K tile (kt); measured (TFLOP/s) 64 / 128 / 256 voxels: 16->16 at
// 128^3 58 / 97 / 78, 48->16 164 / 220 / 210, 64->64 at 32^3 180 / 254 / 277,
// 96->32 at 64^3 328 / 261 / 413, 64->256 at 64^3 451 / 537 / 461: 256 for
// Cin >= 96 with Cout <= 64 (when the stages fit), else 128

__device__ __forceinline__ uint64_t umma_sdesc_mn(uint32_t saddr, uint32_t row_bytes, uint32_t lbo) {
    const uint64_t layout = row_bytes == 128 ? 2 : row_bytes == 64 ? 4 : 6;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(((8 * row_bytes) >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (layout << 61);
}

__global__ void __launch_bounds__(128) k_conv3d_wgrad_tma(const __grid_constant__ CUtensorMap dymap,
                                                           const __grid_constant__ CUtensorMap xmap, float* __restrict__ dw,
                                                           const Vol V, int cin, int cout, const TmaWgrad G) {
    extern __shared__ unsigned char wg_smem_raw[];
    const uint32_t raw = smem_u32(wg_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gen = wg_smem_raw + (base - raw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int S = G.stages;
    uint64_t* full = reinterpret_cast<uint64_t*>(gen + S * G.stage_bytes);
    uint64_t* empty = full + S;
    uint64_t* acc_full = empty + S;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);
    int* failed = reinterpret_cast<int*>(tmem_slot + 1);
    int* issued = failed + 1;
    int* consumed = failed + 2;

    const int part = blockIdx.x, mt = blockIdx.y, n0 = blockIdx.z * 256;
    const int N = min(256, cin - n0);
    // M tile: taps tap0 .. tap0 + taps_per_m - 1 (those < 27) of channels co0 .. co0 + mrows / taps - 1
    const int tap0 = G.co_blocks > 1 ? mt / G.co_blocks : mt * G.taps_per_m;
    const int co0 = G.co_blocks > 1 ? (mt % G.co_blocks) * 128 : 0;
    const int ntaps = G.co_blocks > 1 ? 1 : min(G.taps_per_m, 27 - tap0);
    const int co_rows = G.co_blocks > 1 ? 128 : cout;   // M rows per tap
    const int a_boxes_per_tap = co_rows / G.wsa;
    const int b_boxes = N / G.wsb;
    const int k_begin = part * G.per_part, k_end = min(G.ktiles, k_begin + G.per_part);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(G.cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 32) {
        for (int s = 0; s < 2 * S + 1; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        *failed = *issued = *consumed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int iters = k_end - k_begin;

    if (t == 0) {   // producer
        asm volatile("prefetch.tensormap [%0];" ::"l"(&dymap) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&xmap) : "memory");
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            if (it >= S && !mbar_wait(smem_u32(empty + s), (uint32_t)((it / S - 1) & 1))) {
                atomicExch(failed, 1);
                break;
            }
            long long kt = k_begin + it;
            const int tx = (int)(kt % G.tiles_x);
            kt /= G.tiles_x;
            const int ty = (int)(kt % G.tiles_y);
            kt /= G.tiles_y;
            const int z = (int)(kt % V.d), b = (int)(kt / V.d);
            const int x0 = tx * G.wt, y0 = ty * G.ht;
            const uint32_t st = base + s * G.stage_bytes, bar = smem_u32(full + s);
            mbar_expect(bar, (uint32_t)(ntaps * a_boxes_per_tap) * G.a_box + (uint32_t)b_boxes * G.b_box);
            for (int q = 0; q < ntaps; ++q) {
                const int tap = tap0 + q;
                for (int j = 0; j < a_boxes_per_tap; ++j)
                    tma_5d(st + (uint32_t)(q * a_boxes_per_tap + j) * G.a_box, &dymap, co0 + j * G.wsa,
                           x0 - (tap % 3 - 1), y0 - ((tap / 3) % 3 - 1), z - (tap / 9 - 1), b, bar);
            }
            for (int j = 0; j < b_boxes; ++j)
                tma_5d(st + G.a_bytes + (uint32_t)j * G.b_box, &xmap, n0 + j * G.wsb, x0, y0, z, b, bar);
            *issued = it + 1;
        }
    } else if (t == 32) {   // MMA issuer
        const uint32_t idesc = umma_idesc(TC_M, N) | (1u << 15) | (1u << 16);   // A and B MN-major
        const uint32_t ra = (uint32_t)G.wsa * 2, rb = (uint32_t)G.wsb * 2;
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            if (!mbar_wait(smem_u32(full + s), (uint32_t)((it / S) & 1))) {
                atomicExch(failed, 1);
                break;
            }
            *consumed = it + 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + s * G.stage_bytes;
            for (int k = 0; k < G.kt / 16; ++k) {   // two 8-row groups per MMA
                const uint64_t ad = umma_sdesc_mn(st + k * 16 * ra, ra, G.a_box);
                const uint64_t bd = umma_sdesc_mn(st + G.a_bytes + k * 16 * rb, rb, G.b_box);
                const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(empty + s)));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(acc_full)));
    }
    __syncwarp();
    bool ok = iters > 0 ? mbar_wait(smem_u32(acc_full), 0) : true;
    __syncthreads();
    ok = ok && *failed == 0;
    if (!__syncthreads_or(!ok)) {
        if (iters > 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int r = warp * 32 + lane;   // M row = (tap, co)
            const int q = r / co_rows, co = co0 + r % co_rows;
            const bool store = q < ntaps;
            float* out = dw + ((long long)co * 27 + tap0 + q) * cin + n0;
            for (int c = 0; c < N; c += 16) {
                uint32_t v[16];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (store)
                    for (int j = 0; j < 16; j += 4)
                        atomicAdd(reinterpret_cast<float4*>(out + c + j),
                                  make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]), __uint_as_float(v[j + 2]),
                                              __uint_as_float(v[j + 3])));
            }
        }
    } else if (t == 0) {
        atomicExch(&g_conv_error, 1);
        for (int it = *consumed; it < *issued; ++it) mbar_wait(smem_u32(full + it % S), (uint32_t)((it / S) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G.cols));
}

bool tma_wgrad_tiles(const Vol& V, int cin, TmaWgrad& G);

// The plan, or false when the shapes are outside the TMA form (Cout not 16,
// 32, 64 or a multiple of 128).
bool tma_wgrad_plan(const Vol& V, int cin, int cout, TmaWgrad& G) {
    G = TmaWgrad{};
    if (cout == 16 || cout == 32 || cout == 64) {
        G.wsa = cout;
        G.taps_per_m = TC_M / cout;
        G.co_blocks = 1;
        G.m_tiles = (27 + G.taps_per_m - 1) / G.taps_per_m;
    } else if (cout % 128 == 0) {
        G.wsa = 64;
        G.taps_per_m = 1;
        G.co_blocks = cout / 128;
        G.m_tiles = 27 * G.co_blocks;
    } else {
        return false;
    }
    G.wsb = cin % 64 == 0 ? 64 : cin % 32 == 0 ? 32 : 16;
    G.n_tiles = (cin + 255) / 256;
    for (int kt : {cin >= 96 && cout <= 64 ? 256 : 128, 128}) {
        G.kt = kt;
        if (tma_wgrad_tiles(V, cin, G)) return true;
    }
    return false;
}

// The K tiling and stages of plan G for its kt; false when they do not fit.
bool tma_wgrad_tiles(const Vol& V, int cin, TmaWgrad& G) {
    const int nmax = cin < 256 ? cin : 256;
    G.wt = 1;
    while (G.wt < V.w && G.wt < G.kt) G.wt <<= 1;
    G.ht = G.kt / G.wt;
    G.tiles_x = (V.w + G.wt - 1) / G.wt;
    G.tiles_y = (V.h + G.ht - 1) / G.ht;
    G.ktiles = G.tiles_x * G.tiles_y * V.d * V.n;
    // enough CTAs for about 8 per SM, each with at least 16 K tiles
    const long long mn = (long long)G.m_tiles * G.n_tiles;
    long long parts = (148LL * 8 + mn - 1) / mn;
    const long long most = (G.ktiles + 15) / 16;
    if (parts > most) parts = most;
    if (parts < 1) parts = 1;
    G.per_part = (int)((G.ktiles + parts - 1) / parts);
    G.parts = (G.ktiles + G.per_part - 1) / G.per_part;
    G.cols = 32;
    while (G.cols < nmax) G.cols <<= 1;
    G.a_box = (uint32_t)G.kt * G.wsa * 2;
    G.b_box = (uint32_t)G.kt * G.wsb * 2;
    G.a_bytes = (uint32_t)TC_M * G.kt * 2;
    G.b_bytes = (uint32_t)nmax * G.kt * 2;
    G.stage_bytes = (G.a_bytes + G.b_bytes + 1023u) & ~1023u;
    G.stages = (int)((72u * 1024u) / G.stage_bytes);
    if (G.stages < 2) G.stages = 2;
    if (G.stages > 8) G.stages = 8;
    G.smem = (size_t)G.stages * G.stage_bytes + (2 * G.stages + 1) * 8 + 16 + 1024;
    if (G.smem < (size_t)G.cols * 400) G.smem = (size_t)G.cols * 400;
    return G.smem <= 227u * 1024u;
}

int launch_fwd_tma(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                   int cin, int cout, void* stream);

// Raises a kernel's dynamic shared-memory limit when a launch needs more than
// was set before on this device (the attribute call costs microseconds, the
// small layers' kernels tens of them).
int ensure_smem(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NICR_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = done[{kernel, dev}];
    if (bytes <= cur) return NICR_OK;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return NICR_ERR_CUDA;
    cur = bytes;
    return NICR_OK;
}

int check_args(long long voxels, int cin, int cout) {
    if (voxels <= 0 || voxels % 64 != 0 || cin <= 0 || cin % 16 != 0 || cout <= 0 || cout % 16 != 0)
        return NICR_ERR_INVALID_ARG;
    return NICR_OK;
}

}  // namespace

extern "C" {

int nicr_conv3d_fwd_tma(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                        void* stream) {
    return launch_fwd_tma(x, w, nullptr, 0, y, n, d, h, w_, cin, cout, stream);
}

int nicr_conv3d_fwd_act(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                        int cin, int cout, void* stream) {
    // measured at 128^3 (TFLOP/s): march / halo block / per-tap TMA
    //   16->16 170 / 145 / 91, 16->32 238 / 167 / 135, 48->16 128 / 138 / 104,
    //   32->32 200 / 131 / 225, 64->64 - / 214 / 677
    MarchConv M;
    if (cin == 16 && march_plan(Vol{n, d, h, w_}, cin, cout, M)) {
        const int rc = nicr_conv3d_fwd_march(x, w, bias, act, y, n, d, h, w_, cin, cout, stream);
        if (rc != NICR_ERR_INVALID_ARG) return rc;
    }
    HaloConv H;
    if (cout <= 32 && cin * cout <= 768 && halo_plan(Vol{n, d, h, w_}, cin, cout, H)) {
        const int rc = nicr_conv3d_fwd_halo(x, w, bias, act, y, n, d, h, w_, cin, cout, stream);
        if (rc != NICR_ERR_INVALID_ARG) return rc;
    }
    return launch_fwd_tma(x, w, bias, act, y, n, d, h, w_, cin, cout, stream);
}

int nicr_conv3d_fwd_halo(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                         int cin, int cout, void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    HaloConv H;
    if (rc != NICR_OK || !x || !w || !y || (act & ~(ACT_RELU | ACT_BF16)) != 0 || !halo_plan(V, cin, cout, H))
        return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const auto enc = conv_map_encoder();
    if (!enc) return NICR_ERR_CUDA;
    CUtensorMap xmap;
    const cuuint64_t dims[5] = {(cuuint64_t)cin, (cuuint64_t)w_, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)n};
    const cuuint64_t str[4] = {(cuuint64_t)cin * 2, (cuuint64_t)w_ * cin * 2, (cuuint64_t)h * w_ * cin * 2,
                               (cuuint64_t)d * h * w_ * cin * 2};
    const cuuint32_t box[5] = {8, HB_ROWS, 3, 3, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, str, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return NICR_ERR_INVALID_ARG;
    if (ensure_smem((const void*)k_conv3d_fwd_halo, H.smem) != NICR_OK)
        return NICR_ERR_CUDA;
    const long long tiles = (long long)H.tiles_x * h * d * n;
    k_conv3d_fwd_halo<<<(unsigned)tiles, 128, H.smem, static_cast<cudaStream_t>(stream)>>>(
        xmap, static_cast<const __nv_bfloat16*>(w), y, bias, act, V, cin, cout, H);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

int nicr_conv3d_fwd_march(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h,
                          int w_, int cin, int cout, void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    MarchConv M;
    if (rc != NICR_OK || !x || !w || !y || (act & ~(ACT_RELU | ACT_BF16)) != 0 || !march_plan(V, cin, cout, M))
        return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const auto enc = conv_map_encoder();
    if (!enc) return NICR_ERR_CUDA;
    CUtensorMap xmap;
    const cuuint64_t dims[5] = {(cuuint64_t)cin, (cuuint64_t)w_, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)n};
    const cuuint64_t str[4] = {(cuuint64_t)cin * 2, (cuuint64_t)w_ * cin * 2, (cuuint64_t)h * w_ * cin * 2,
                               (cuuint64_t)d * h * w_ * cin * 2};
    const cuuint32_t box[5] = {8, HB_ROWS, 1, 3, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, str, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return NICR_ERR_INVALID_ARG;
    if (ensure_smem((const void*)k_conv3d_fwd_march, M.smem) != NICR_OK)
        return NICR_ERR_CUDA;
    const long long blocks = (long long)M.tiles_x * M.ysplit * d * n;
    k_conv3d_fwd_march<<<(unsigned)blocks, 128, M.smem, static_cast<cudaStream_t>(stream)>>>(
        xmap, static_cast<const __nv_bfloat16*>(w), y, bias, act, V, cin, cout, M);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

}  // extern "C"

namespace {

int launch_fwd_tma(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                   int cin, int cout, void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !w || !y || (act & ~(ACT_RELU | ACT_BF16)) != 0)
        return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const auto enc = conv_map_encoder();
    if (!enc) return NICR_ERR_CUDA;
    const TmaConv C = tma_conv_plan(V, cin, cout);
    const CUtensorMapSwizzle swz = C.kc == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : C.kc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUtensorMap xmap, wmap;
    {   // x: (c, w, h, d, n), boxes {KC, Wt, Ht, 1, 1}
        const cuuint64_t dims[5] = {(cuuint64_t)cin, (cuuint64_t)w_, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)n};
        const cuuint64_t str[4] = {(cuuint64_t)cin * 2, (cuuint64_t)w_ * cin * 2, (cuuint64_t)h * w_ * cin * 2,
                                   (cuuint64_t)d * h * w_ * cin * 2};
        const cuuint32_t box[5] = {(cuuint32_t)C.kc, (cuuint32_t)C.wt, (cuuint32_t)C.ht, 1, 1};
        if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, str, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return NICR_ERR_INVALID_ARG;
    }
    {   // w: (ci, tap, co), boxes {KC, 1, min(cout, 256)}
        const cuuint64_t dims[3] = {(cuuint64_t)cin, 27, (cuuint64_t)cout};
        const cuuint64_t str[2] = {(cuuint64_t)cin * 2, (cuuint64_t)27 * cin * 2};
        const cuuint32_t box[3] = {(cuuint32_t)C.kc, 1, (cuuint32_t)(cout < 256 ? cout : 256)};
        if (enc(&wmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(w), dims, str, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return NICR_ERR_INVALID_ARG;
    }
    if (ensure_smem((const void*)k_conv3d_fwd_tma, C.smem) != NICR_OK)
        return NICR_ERR_CUDA;
    const long long tiles = (long long)C.tiles_x * C.tiles_y * d * n;
    const dim3 grid((unsigned)tiles, (unsigned)((cout + 255) / 256));
    k_conv3d_fwd_tma<<<grid, 128, C.smem, static_cast<cudaStream_t>(stream)>>>(xmap, wmap, y, bias, act, V, cin,
                                                                                   cout, C);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

}  // namespace

extern "C" {

int nicr_conv3d_fwd(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                    void* stream) {
    const int rc = nicr_conv3d_fwd_act(x, w, nullptr, 0, y, n, d, h, w_, cin, cout, stream);
    if (rc != NICR_ERR_INVALID_ARG || check_args((long long)n * d * h * w_, cin, cout) != NICR_OK || !x || !w || !y)
        return rc;
    // a tensor map the driver refused: the gathering form
    return nicr_conv3d_fwd_gather(x, w, y, n, d, h, w_, cin, cout, stream);
}

int nicr_conv3d_fwd_gather(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                           void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !w || !y) return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const int cmax = cout < 256 ? cout : 256;
    int kc = 64;   // channels per chunk: the largest of 64, 48, 32, 16 dividing Cin
    while (cin % kc != 0) kc -= 16;
    const size_t stage = ((size_t)(TC_M + cmax) * kc * 2 + 1023) / 1024 * 1024;
    int cols = 32;   // TMEM columns: a power of two >= N
    while (cols < cmax) cols <<= 1;
    // at least cols x 400 bytes of shared memory per CTA, so that the CTAs
    // resident on one SM never ask for more than its 512 TMEM columns
    size_t smem = TC_STAGES * stage + 64;
    if (smem < (size_t)cols * 400) smem = (size_t)cols * 400;
    if (ensure_smem((const void*)k_conv3d_fwd_tc, smem) != NICR_OK)
        return NICR_ERR_CUDA;
    const dim3 grid((unsigned)((V.voxels() + TC_M - 1) / TC_M), (unsigned)((cout + 255) / 256));
    k_conv3d_fwd_tc<<<grid, 128, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), y, V, cin, cout, kc, cols);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

int nicr_conv3d_fwd_mma_sync(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                             void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !w || !y) return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    const dim3 grid((unsigned)(V.voxels() / BM), (unsigned)((cout + BN - 1) / BN));
    k_conv3d_fwd<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), y, V, cin, cout);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

int nicr_conv3d_wgrad_tma(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                          void* stream) {
    const Vol V{n, d, h, w_};
    const int rc = check_args(V.voxels(), cin, cout);
    if (rc != NICR_OK || !x || !dy || !dw) return rc != NICR_OK ? rc : NICR_ERR_INVALID_ARG;
    TmaWgrad G;
    if (!tma_wgrad_plan(V, cin, cout, G)) return NICR_ERR_INVALID_ARG;
    const auto enc = conv_map_encoder();
    if (!enc) return NICR_ERR_CUDA;
    auto swz = [](int ws) {
        return ws == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : ws == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    };
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUtensorMap dymap, xmap;
    // (c, w, h, d, n) views of dy (Cout channels) and x (Cin channels), boxes {Ws, Wt, Ht, 1, 1}
    auto encode = [&](CUtensorMap* m, const void* p, int c, int ws) {
        const cuuint64_t dims[5] = {(cuuint64_t)c, (cuuint64_t)w_, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)n};
        const cuuint64_t str[4] = {(cuuint64_t)c * 2, (cuuint64_t)w_ * c * 2, (cuuint64_t)h * w_ * c * 2,
                                   (cuuint64_t)d * h * w_ * c * 2};
        const cuuint32_t box[5] = {(cuuint32_t)ws, (cuuint32_t)G.wt, (cuuint32_t)G.ht, 1, 1};
        return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(p), dims, str, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz(ws), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    if (!encode(&dymap, dy, cout, G.wsa) || !encode(&xmap, x, cin, G.wsb)) return NICR_ERR_INVALID_ARG;
    if (ensure_smem((const void*)k_conv3d_wgrad_tma, G.smem) != NICR_OK)
        return NICR_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(dw, 0, sizeof(float) * (size_t)cout * 27 * cin, s) != cudaSuccess) return NICR_ERR_CUDA;
    const dim3 grid((unsigned)G.parts, (unsigned)G.m_tiles, (unsigned)G.n_tiles);
    k_conv3d_wgrad_tma<<<grid, 128, G.smem, s>>>(dymap, xmap, dw, V, cin, cout, G);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}

int nicr_conv3d_wgrad(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                      void* stream) {
    const int rc = nicr_conv3d_wgrad_tma(x, dy, dw, n, d, h, w_, cin, cout, stream);
    if (rc != NICR_ERR_INVALID_ARG || check_args((long long)n * d * h * w_, cin, cout) != NICR_OK || !x || !dy || !dw)
        return rc;
    // Cout outside the TMA form, or tensor maps the driver refused
    return nicr_conv3d_wgrad_mma_sync(x, dy, dw, n, d, h, w_, cin, cout, stream);
}

int nicr_conv3d_wgrad_mma_sync(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
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

int nicr_conv3d_error(int* flag) {
    if (!flag) return NICR_ERR_INVALID_ARG;
    const int zero = 0;
    if (cudaMemcpyFromSymbol(flag, g_conv_error, sizeof(int)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_conv_error, &zero, sizeof(int)) != cudaSuccess)
        return NICR_ERR_CUDA;
    return NICR_OK;
}

}  // extern "C"
