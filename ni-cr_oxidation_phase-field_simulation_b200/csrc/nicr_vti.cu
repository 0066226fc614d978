// The seven point-data arrays of a 3D VTI frame (write_vti, 3S:238-334:
// phi, conc_O, conc_Cr, mu_O, mu_Cr, grain_sum, GB_mask), computed on the GPU
// in the file's order (X fastest) and type (Float32 or Float64), so that only
// the finished arrays cross PCIe and the host does nothing but compress and
// write. The state is stored X slowest: each CTA transposes a 32 x 32 tile of
// one (X, Z) plane at fixed Y through shared memory, reading and writing
// coalesced. Values are the reference's expressions in FP64 (grain_sum:
// sum_g (g+1) eta_g in g order, or grain * (1 - h(phi)); 3S:534-545), then
// rounded to the output type as static_cast does on the host. A Float32 value
// that is finite but outside the float range sets the array's bit in *range
// (the reference refuses to write such a frame).
#include <cuda_runtime.h>

#include <cfloat>

#include "nicr_kernels.h"
#include "nicr_physics.h"

namespace nicr {
namespace {

template <class T>
__global__ void __launch_bounds__(256) k_vti_arrays(const VtiArgs a, T* __restrict__ out, unsigned* range) {
    __shared__ double tile[32][33];
    const Grid& g = a.g;
    const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32, j = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long n = (long long)g.nx * g.na * g.nb;
    for (int arr = 0; arr < 7; ++arr) {
        // read: k fastest (coalesced), value of array `arr` at (i, j, k)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int i = i0 + ty + 8 * r, k = k0 + tx;
            double v = 0.;
            if (i < g.nx && k < g.nb) {
                const long long q = (long long)i * g.plane + (long long)j * g.pb + k;
                switch (arr) {
                    case 0: v = a.p[q]; break;
                    case 1: v = a.o[q]; break;
                    case 2: v = a.cr[q]; break;
                    case 3: v = a.muO[q]; break;
                    case 4: v = a.muCr[q]; break;
                    case 5:
                        if (a.has_eta) {
                            double s = 0.;
                            for (int e = 0; e < a.neta; ++e) s += double(e + 1) * a.eta[(long long)e * g.nstore + q];
                            v = s;
                        } else {
                            v = a.grain[q] * (1. - h(a.p[q]));
                        }
                        break;
                    default: v = a.gb[q]; break;
                }
            }
            tile[ty + 8 * r][tx] = v;
        }
        __syncthreads();
        // write: i fastest (coalesced), X-fastest file order ((k * ny + j) * nx + i)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int k = k0 + ty + 8 * r, i = i0 + tx;
            if (i < g.nx && k < g.nb) {
                const double v = tile[tx][ty + 8 * r];
                if (sizeof(T) == 4 && isfinite(v) && fabs(v) > (double)FLT_MAX) atomicOr(range, 1u << arr);
                out[(long long)arr * n + ((long long)k * g.na + j) * g.nx + i] = static_cast<T>(v);
            }
        }
        __syncthreads();
    }
}

}  // namespace

void launch_vti_arrays(const VtiArgs& a, void* out, bool f64, unsigned* range, cudaStream_t stream) {
    const Grid& g = a.g;
    const dim3 grid((g.nb + 31) / 32, (g.nx + 31) / 32, g.na), block(32, 8);
    if (f64) k_vti_arrays<double><<<grid, block, 0, stream>>>(a, static_cast<double*>(out), range);
    else k_vti_arrays<float><<<grid, block, 0, stream>>>(a, static_cast<float*>(out), range);
}

}  // namespace nicr
