// nicr_step_noalloc: one step of c_O, c_Cr and phi on caller-owned device
// arrays, in the FP64 form the configuration selects (the bit-identical
// drop-in form or the reciprocal form), for callers that must not allocate
// device memory.
//
// Who needs it: codes that embed the step inside their own time loop and own
// every byte of device memory through their own pool (a coupled multiphysics
// driver that budgets HBM up front), code that runs where the CUDA memory API
// may not be called (host functions enqueued with cudaLaunchHostFunc, some
// real-time loops), and callers that must not grow the memory footprint after
// start-up. The handle API allocates its buffers in nicr_create; this entry
// point needs none: the caller passes the inputs and outputs, and the step's
// scratch (per-CTA budget partial sums and the trial status word) lives in
// the file-scope device array below.
//
// The scratch array is shared by every call in the process on a given device,
// and keeps the last call's contents; each call first clears the status word.
// Calls whose kernels overlap on the GPU (different streams, no ordering)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/nicr.h"
#include "nicr_kernels.h"
#include "nicr_physics.h"

namespace {

// Largest step grid the scratch array serves: 8192 CTAs of the step kernel.
// params_for lengthens the X chunk (planes per CTA) until the grid fits, so
// every grid with at most 8192 step tiles per X plane is served (3D tiles of
// 8 rows x 32 columns: ceil(ny/8)*ceil(nz/32) <= 8192; 2D tiles of 128
// columns: ceil(ny/128) <= 8192).
constexpr int kMaxCtas = 8192;
struct Scratch {
    nicr::Status status;
    unsigned char pad[256 - sizeof(nicr::Status)];
    nicr::StepPartial partials[kMaxCtas];
};
// 256-byte aligned, ~768 KB; every GPU that loads the library holds it until exit.
static __device__ __align__(256) Scratch g_scratch;

// Device addresses of g_scratch, resolved once per device (host code must not
// use the symbol itself: on the host it is only a stand-in, not a device address).
constexpr int kMaxDevices = 64;
Scratch* g_addr[kMaxDevices] = {};
std::mutex g_mu;

__global__ void k_status_clear(nicr::Status* st) {
    st->err_key = nicr::ERR_NONE;
    st->failed = 0;
    st->timeout = 0;
    st->failed_step = -1;
    st->slot_err[0] = st->slot_err[1] = nicr::ERR_NONE;
}

// Reduces the per-CTA partials in block order (deterministic) into the
// caller's result struct.
__global__ void k_step_result(const nicr::StepPartial* __restrict__ partials, int nblocks, const nicr::Status* st,
                              nicr_step_result* out) {
    __shared__ nicr::DD sdd[32][5];
    __shared__ long long scnt[32];
    nicr::DD acc[5] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    long long clipped = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        for (int q = 0; q < 5; ++q) acc[q] = nicr::dd_add(acc[q], nicr::DD{partials[b].s[q][0], partials[b].s[q][1]});
        clipped += partials[b].clipped;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int off = 16; off > 0; off >>= 1) {
        for (int q = 0; q < 5; ++q)
            acc[q] = nicr::dd_add(acc[q], nicr::DD{__shfl_down_sync(0xffffffffu, acc[q].hi, off),
                                                   __shfl_down_sync(0xffffffffu, acc[q].lo, off)});
        clipped += __shfl_down_sync(0xffffffffu, clipped, off);
    }
    if (lane == 0) {
        for (int q = 0; q < 5; ++q) sdd[w][q] = acc[q];
        scnt[w] = clipped;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 5; ++q) acc[q] = sdd[0][q];
        clipped = scnt[0];
        for (int ww = 1; ww < nw; ++ww) {
            for (int q = 0; q < 5; ++q) acc[q] = nicr::dd_add(acc[q], sdd[ww][q]);
            clipped += scnt[ww];
        }
        double* dst[5] = {out->ckO, out->ckCr, out->clipO, out->clipCr, out->bcO};
        for (int q = 0; q < 5; ++q) { dst[q][0] = acc[q].hi; dst[q][1] = acc[q].lo; }
        out->clipped = clipped;
        out->trial_key = st->err_key;
    }
}

// Step parameters from a configuration, for packed arrays (column pitch = nz
// in 3D, ny in 2D): the same values and the same X chunking as the handle API.
nicr::StepParams params_for(const nicr_config& c) {
    using namespace nicr;
    StepParams sp{};
    const int dim = c.dim;
    Grid& g = sp.g;
    g.dim = dim;
    g.nx = c.nx;
    g.na = dim == 3 ? c.ny : 1;
    g.nb = dim == 3 ? c.nz : c.ny;
    g.pb = g.nb;
    g.plane = (long long)g.na * g.pb;
    g.ncells = (long long)g.nx * g.na * g.nb;
    g.nstore = (long long)g.nx * g.plane;
    const bool has_eta = c.grain_evolution && c.grains;
    const EtaCoef ec = eta_coef(c.gb_fwhm_grid, c.dx, c.eta_W, c.eta_kappa, c.eta_oxide_penalty);
    sp.dx = c.dx;
    sp.da = c.dy;
    sp.db = dim == 3 ? c.dz : c.dy;
    sp.dt = c.dt;
    sp.dxdx = c.dx * c.dx;
    sp.dada = c.dy * c.dy;
    sp.dbdb = dim == 3 ? c.dz * c.dz : c.dy * c.dy;
    sp.v_dxdx = make_divc(sp.dxdx);
    sp.v_dada = make_divc(sp.dada);
    sp.v_dbdb = make_divc(sp.dbdb);
    sp.v_dx = make_divc(sp.dx);
    sp.v_da = make_divc(sp.da);
    sp.v_db = make_divc(sp.db);
    sp.v_dt = make_divc(sp.dt);
    sp.dtL = c.dt * Phys::L;
    sp.layer_o = c.layer_o;
    sp.gbm1_o = c.gb_factor_o - 1.;
    sp.gbm1_cr = c.gb_factor_cr - 1.;
    sp.mu_res = c.mu_res;
    sp.surface_c_ref = c.surface_c_ref;
    sp.eta_W = c.eta_W;
    sp.eta_A = ec.A;
    sp.eta_K = ec.K;
    sp.dt_etaL = c.dt * c.eta_L;
    sp.eta_scale = ec.scale;
    sp.bc = c.bc;
    sp.ck = c.ck;
    sp.bounds = c.bounds;
    sp.o_on = c.oxygen_diffusion ? 1 : 0;
    sp.grains = c.grains ? 1 : 0;
    sp.phi_eta = has_eta ? 1 : 0;
    sp.inlet = (c.bc == NICR_BC_CONCENTRATION && c.oxygen_diffusion) ? 1 : 0;
    sp.fast = c.precision == NICR_FP64_FAST ? 1 : 0;
    sp.xchunk = choose_xchunk(g);
    whole_domain_range(sp);
    // Longer X chunks mean fewer CTAs; the fields do not depend on the chunk
    // (budget partial sums group differently, ~1e-16 relative).
    while (step_main_blocks(sp) > kMaxCtas && sp.xchunk < g.nx) sp.xchunk = std::min(g.nx, 2 * sp.xchunk);
    return sp;
}

}  // namespace

extern "C" int nicr_step_noalloc(const nicr_config* cfg, const double* o, const double* cr, const double* p,
                                 const double* gb, const double* eta_s2, double* o_next, double* cr_next,
                                 double* p_next, nicr_step_result* result, void* stream) {
    if (!cfg || (cfg->dim != 2 && cfg->dim != 3) || cfg->nx < 3 || cfg->ny < 3 || (cfg->dim == 3 && cfg->nz < 3))
        return NICR_ERR_INVALID_ARG;
    // the same arithmetic forms as nicr_create accepts
    if (cfg->precision != NICR_FP64 && cfg->precision != NICR_FP64_FAST) return NICR_ERR_INVALID_ARG;
    const nicr::StepParams sp = params_for(*cfg);
    // reject sizes beyond the scratch array before touching the device
    if (nicr::step_main_blocks(sp) > kMaxCtas) return NICR_ERR_INVALID_ARG;
    if (!o || !cr || !p || !o_next || !cr_next || !p_next || !result) return NICR_ERR_INVALID_ARG;
    if (cfg->grains && !gb) return NICR_ERR_INVALID_ARG;
    if (cfg->grain_evolution && cfg->grains && !eta_s2) return NICR_ERR_INVALID_ARG;
    // An error already pending on this thread belongs to the caller's earlier
    // work: leave it in place for the caller and enqueue nothing. Past this
    // point every launch error read (and cleared) below is this call's own.
    if (cudaPeekAtLastError() != cudaSuccess) return NICR_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NICR_ERR_NO_DEVICE;
    Scratch* s = nullptr;
    {
        // first call on this device: resolve the array's device address
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || !ptr) return NICR_ERR_CUDA;
            g_addr[dev] = static_cast<Scratch*>(ptr);
        }
        s = g_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_status_clear<<<1, 1, 0, st>>>(&s->status);
    int nb = 0;
    nicr::launch_step_main(sp, o, cr, p, cfg->grains ? gb : nullptr, eta_s2, o_next, cr_next, p_next, s->partials,
                           &s->status, st, &nb);
    k_step_result<<<1, 256, 0, st>>>(s->partials, nb, &s->status, result);
    return cudaGetLastError() == cudaSuccess ? NICR_OK : NICR_ERR_CUDA;
}
