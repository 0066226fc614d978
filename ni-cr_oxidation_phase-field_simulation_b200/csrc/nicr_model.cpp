// Host orchestration of one GPU-resident domain (see nicr_model.h).
#include "nicr_model.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <sstream>
#include <iomanip>
#include <thread>

namespace nicr {

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(NICR_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

namespace {

// Runs fn(begin, end) over [0, n) on the host cores.
template <class Fn>
void parallel_for(long long n, Fn fn) {
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n < 1 << 16) nt = 1;
    std::vector<std::thread> th;
    const long long chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const long long b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=] { fn(b, e); });
    }
    for (auto& t : th) t.join();
}

int bounded_reach_h(double radius, int n) { return radius >= n ? n : int(std::ceil(radius)); }

}  // namespace

double* Model::dalloc(size_t n) { return dalloc_t<double>(n); }
template <class T>
T* Model::dalloc_t(size_t n) {
    T* p = nullptr;
    check_cuda(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    dev_bytes += std::max<size_t>(n, 1) * sizeof(T);
    return p;
}

Model::Model(const nicr_config& cfg, const SlabSpec* slab) : c(cfg), dim(cfg.dim) {
    if (dim != 2 && dim != 3) throw Error(NICR_ERR_INVALID_ARG, "dim must be 2 or 3");
    if (dim == 3 && (c.nx < 3 || c.ny < 3 || c.nz < 3 || c.nx > INT_MAX - 2 || c.ny > INT_MAX - 2 || c.nz > INT_MAX - 2))
        throw Error(NICR_ERR_INVALID_ARG, "3D grid dimensions must lie in [3, INT_MAX-2].");
    if (dim == 2 && (c.nx < 3 || c.ny < 3))
        throw Error(NICR_ERR_INVALID_ARG, "Invalid parameter bounds (Ksp nucleation period must be >= dt).");
    if (dim == 2) c.nz = 1;
    int hlo = 0, hhi = 0;
    if (slab) {
        if (dim != 3) throw Error(NICR_ERR_INVALID_ARG, "the slab form is 3D only");
        const SlabSpec& q = *slab;
        if (q.halo < 2 || q.x0 < 0 || q.x1 > c.nx || q.x1 - q.x0 < q.halo || (q.x0 > 0 && q.x0 < q.halo) ||
            (q.x1 < c.nx && c.nx - q.x1 < q.halo))
            throw Error(NICR_ERR_INVALID_ARG, "slab planes must be at least the halo width and within the domain");
        is_slab = true;
        hlo = q.x0 > 0 ? q.halo : 0;
        hhi = q.x1 < c.nx ? q.halo : 0;
        x_off = q.x0 - hlo;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(NICR_ERR_NO_DEVICE, "no CUDA device is available");
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");

    g.dim = dim;
    g.nx = is_slab ? slab->x1 - slab->x0 + hlo + hhi : c.nx;
    g.na = dim == 3 ? c.ny : 1;
    g.nb = dim == 3 ? c.nz : c.ny;
    g.pb = (g.nb + 7) / 8 * 8;
    g.plane = (long long)g.na * g.pb;
    g.ncells = (long long)g.nx * g.na * g.nb;
    g.nstore = (long long)g.nx * g.plane;

    has_eta = c.grain_evolution && c.grains;
    advance_eta = has_eta && (dim == 2 || c.eta_L > 0.);
    ec = eta_coef(c.gb_fwhm_grid, c.dx, c.eta_W, c.eta_kappa, c.eta_oxide_penalty);
    next_nucleation = c.nucleation_period;

    sp.g = g;
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
    // the inlet layer is domain plane 0 (a slab above it only reads it)
    sp.inlet = (c.bc == NICR_BC_CONCENTRATION && c.oxygen_diffusion && x_off == 0) ? 1 : 0;
    if (c.precision != NICR_FP64 && c.precision != NICR_FP64_FAST)
        throw Error(NICR_ERR_INVALID_ARG, "precision must be NICR_FP64 or NICR_FP64_FAST");
    sp.fast = c.precision == NICR_FP64_FAST ? 1 : 0;
    whole_domain_range(sp);
    if (is_slab) {
        sp.x_lo = hlo;
        sp.x_hi = hlo + (slab->x1 - slab->x0);
        sp.cell_off = (long long)x_off * g.na * g.nb;
        sp.key_ncells = (long long)c.nx * g.na * g.nb;
        sp.err_slot = 0;
    }
    sp.xchunk = choose_xchunk(own_grid());

    try {
        const size_t ns = (size_t)g.nstore;
        for (int q = 0; q < 2; ++q) { o_[q] = dalloc(ns); cr_[q] = dalloc(ns); p_[q] = dalloc(ns); }
        gb_[0] = dalloc(ns);
        check_cuda(cudaMemsetAsync(gb_[0], 0, ns * 8, stream), "memset");
        if (advance_eta) gb_[1] = dalloc(ns);
        if (has_eta) { s2_[0] = dalloc(ns); if (advance_eta) s2_[1] = dalloc(ns); }
        grain = dalloc(ns);
        if (dim == 2) { gb_initial = dalloc(ns); if (has_eta) { pairs = dalloc(ns); check_cuda(cudaMemsetAsync(pairs, 0, ns * 8, stream), "memset"); } }
        partial_cap = std::max(step_main_blocks(sp), 148 * 4) + 8;
        partials = dalloc_t<StepPartial>(partial_cap);
        st = dalloc_t<Status>(1);
        bud = dalloc_t<DevBudget>(1);
        diag_part = dalloc_t<DiagOut>(148 * 4 + 8);
        diag_out = dalloc_t<DiagOut>(1);
        red_out = dalloc_t<StepPartial>(1);
        check_cuda(cudaMallocHost(&h_st, sizeof(Status)), "cudaMallocHost");
        check_cuda(cudaMemsetAsync(bud, 0, sizeof(DevBudget), stream), "memset");
        Status s0{ERR_NONE, 0, 0, -1, 0, {ERR_NONE, ERR_NONE}};
        *h_st = s0;
        check_cuda(cudaMemcpyAsync(st, h_st, sizeof(Status), cudaMemcpyHostToDevice, stream), "memcpy");

        voronoi();
        InitParams I = init_params();
        I.bulk_cr = c.bulk_cr; I.layer_o = c.layer_o; I.inlet_layer = c.bc == NICR_BC_CONCENTRATION;
        launch_init_fields(I, o_[0], cr_[0], p_[0], stream);
        if (dim == 2) check_cuda(cudaMemcpyAsync(gb_initial, gb_[0], ns * 8, cudaMemcpyDeviceToDevice, stream), "memcpy");
        reset_inventory();
        if (c.nucleation == NICR_NUC_CENTER) init_center_seed();
        if (has_eta) {
            const int nfields = c.eta_colours > 0 ? c.eta_colours : (int)(seeds.size() / dim);
            if (nfields > c.max_eta_fields)
                throw Error(NICR_ERR_INVALID_ARG, dim == 3 ? "Too many eta fields; check --max-eta-fields and memory."
                                                           : "Too many eta fields. Increase --max-eta-fields only after checking memory, or use --grain-evolution off.");
            if (c.eta_colours > 0) {
                if (dim != 3) throw Error(NICR_ERR_INVALID_ARG, "--eta-colours is 3D only");
                grain_adjacency();
                alloc_eta(c.eta_colours);
                // a slab sees part of the adjacency: its group colours the union
                if (!is_slab) {
                    seed_colour = colour_grains(adjacency, (int)(seeds.size() / 3), c.eta_colours);
                    init_eta_coloured();
                }
            } else {
                init_eta();
            }
            if (dim == 3) grain_retained = false;
        }
        if (c.nucleation == NICR_NUC_KSP) setup_ksp();
        if (has_eta) eta_mask_now();
        // the one-pass step runs one 16 x 32 tile per SM: its own chunk choice
        if (onepass_step()) set_xchunk(choose_xchunk_fused(g));
        check_cuda(cudaStreamSynchronize(stream), "init");
        check_cuda(cudaGetLastError(), "init kernels");
    } catch (...) {
        release();
        throw;
    }
}

Model::~Model() {
    output_writer.reset();   // finishes pending output before the buffers go
    release();
}

void Model::release() {
    if (stream) cudaStreamSynchronize(stream);
    double* bufs[] = {o_[0], o_[1], cr_[0], cr_[1], p_[0], p_[1], gb_[0], gb_[1], s2_[0], s2_[1], eta_[0], eta_[1],
                      grain, pairs, gb_initial, muO, muCr, mo, mc};
    for (double* b : bufs) if (b) cudaFree(b);
    void* others[] = {partials, st, bud, diag_part, diag_out, red_out, kres, d_shadow, d_ball, d_hyp, agree, ticket,
                      kw.flag, kw.blocked, kw.counts, kw.list, kw.total, gw.cells, gw.parts, gw.amount_parts,
                      g_out, g_amount, g_cells};
    for (void* b : others) if (b) cudaFree(b);
    if (h_st) cudaFreeHost(h_st);
    for (cudaEvent_t e : prof_pool) cudaEventDestroy(e);
    prof_pool.clear();
    for (auto& q : pair_graphs)
        if (q.exec) { cudaGraphExecDestroy(q.exec); q.exec = nullptr; }
    if (stream && owns_stream) cudaStreamDestroy(stream);
    std::memset(o_, 0, sizeof o_); std::memset(cr_, 0, sizeof cr_); std::memset(p_, 0, sizeof p_);
    std::memset(gb_, 0, sizeof gb_); std::memset(s2_, 0, sizeof s2_); std::memset(eta_, 0, sizeof eta_);
    grain = pairs = gb_initial = muO = muCr = mo = mc = nullptr;
    partials = nullptr; st = nullptr; bud = nullptr; diag_part = diag_out = nullptr; red_out = nullptr; kres = nullptr;
    d_shadow = d_ball = nullptr; d_hyp = nullptr; kw = KspWork{}; h_st = nullptr; stream = nullptr; agree = nullptr; ticket = nullptr;
    gw = GrainWork{}; g_out = nullptr; g_amount = nullptr; g_cells = nullptr;
}

void Model::sync() { check_cuda(cudaStreamSynchronize(stream), "stream"); }

void Model::copy_out(const double* d, double* host) {
    check_cuda(cudaMemcpy2DAsync(host, (size_t)g.nb * 8, d, (size_t)g.pb * 8, (size_t)g.nb * 8, (size_t)g.nx * g.na,
                                 cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
}
void Model::copy_in(double* d, const double* host) {
    check_cuda(cudaMemcpy2DAsync(d, (size_t)g.pb * 8, host, (size_t)g.nb * 8, (size_t)g.nb * 8, (size_t)g.nx * g.na,
                                 cudaMemcpyHostToDevice, stream), "H2D");
    sync();
}

// ------------------------------------------------------------------ init
// Voronoi grains (3S:407-467, 2D:233-291). Seeds come from libstdc++'s
// mt19937_64 + uniform_real_distribution exactly as in the reference.
void Model::voronoi() {
    seeds.clear();
    volumes.clear();
    const size_t ns = (size_t)g.nstore;
    if (!c.grains) {
        seeds.push_back(0.5 * c.nx);
        seeds.push_back(0.5 * c.ny);
        if (dim == 3) seeds.push_back(0.5 * c.nz);
        volumes.push_back(is_slab ? own_grid().ncells : dim == 3 ? (long long)(c.nx * c.ny * c.nz) : (long long)(c.nx * c.ny));
        std::vector<double> ones((size_t)g.ncells, 1.);
        copy_in(grain, ones.data());
        check_cuda(cudaMemsetAsync(gb_[0], 0, ns * 8, stream), "memset");
        return;
    }
    int ng;
    if (dim == 3) {
        const double volume = double(c.nx) * c.ny * c.nz;
        const double ng_real = 6. * volume / (PI * std::pow(c.grain_diameter_grid, 3));
        if (!std::isfinite(ng_real) || ng_real > volume + .5) throw Error(NICR_ERR_INVALID_ARG, "Too many Voronoi sites for this grid.");
        ng = std::max(1, int(std::llround(ng_real)));
        if (ng > volume) throw Error(NICR_ERR_INVALID_ARG, "Too many Voronoi sites for this grid.");
        if (has_eta && c.eta_colours <= 0 && ng > c.max_eta_fields)
            throw Error(NICR_ERR_INVALID_ARG, "3D grain count exceeds --max-eta-fields; increase grain diameter or check memory before increasing the limit.");
    } else {
        const double domain_area = double(c.nx) * c.ny;
        ng = std::max(1, int(std::llround(4. * domain_area / (PI * c.grain_diameter_grid * c.grain_diameter_grid))));
        if (ng > c.nx * c.ny) throw Error(NICR_ERR_INVALID_ARG, "Too many Voronoi sites for this grid.");
    }
    std::mt19937_64 rng(c.random_seed);
    std::uniform_real_distribution<double> ux(0., double(c.nx)), uy(0., double(c.ny)), uz(0., double(c.nz));
    for (int q = 0; q < ng; ++q) {
        const double x = ux(rng), y = uy(rng);
        seeds.push_back(x);
        seeds.push_back(y);
        if (dim == 3) seeds.push_back(uz(rng));
    }
    const int D = dim;
    if (D == 3) {
        if (c.left_edge_sites < 0 || c.left_edge_sites > std::min(ng, c.ny * c.nz))
            throw Error(NICR_ERR_INVALID_ARG, "--left-face-sites must be between 0 and min(volume-based site count, ny*nz).");
        if (c.left_edge_sites > 0) {  // 3S:430-449
            const int n = c.left_edge_sites;
            int rows = std::clamp(int(std::llround(std::sqrt(double(n) * c.ny / c.nz))), 1, std::min(n, c.ny));
            rows = std::max(rows, (n + c.nz - 1) / c.nz);
            std::uniform_real_distribution<double> unit(0., 1.);
            const int phaseY = std::min(c.ny - 1, int(unit(rng) * c.ny));
            const int phaseZ = std::min(c.nz - 1, int(unit(rng) * c.nz));
            int q = 0;
            for (int r = 0; r < rows; ++r) {
                const int cols = n / rows + (r < n % rows ? 1 : 0);
                const int yy = (phaseY + int(static_cast<long long>(r) * c.ny / rows)) % c.ny;
                for (int k = 0; k < cols; ++k) {
                    const int zz = (phaseZ + int(static_cast<long long>(k) * c.nz / cols)) % c.nz;
                    seeds[3 * q] = 0.05 + 0.4 * unit(rng);
                    seeds[3 * q + 1] = yy + 0.5;
                    seeds[3 * q + 2] = zz + 0.5;
                    ++q;
                }
            }
            for (int s = n; s < ng; ++s) seeds[3 * s] = 1.5 + (c.nx - 1.5) * (seeds[3 * s] / c.nx);
        }
    } else {
        if (c.left_edge_sites < 0 || c.left_edge_sites > std::min(ng, c.ny))
            throw Error(NICR_ERR_INVALID_ARG, "--left-edge-sites must be between 0 and min(area-based site count, ny).");
        if (c.left_edge_sites > 0) {  // 2D:251-265
            std::uniform_real_distribution<double> unit(0., 1.);
            const int phase = std::min(c.ny - 1, int(unit(rng) * c.ny));
            for (int k = 0; k < c.left_edge_sites; ++k) {
                const int row = (phase + int((static_cast<long long>(k) * c.ny) / c.left_edge_sites)) % c.ny;
                seeds[2 * k] = 0.05 + 0.4 * unit(rng);
                seeds[2 * k + 1] = row + 0.5;
            }
            for (int k = c.left_edge_sites; k < ng; ++k) seeds[2 * k] = 1.5 + (c.nx - 1.5) * (seeds[2 * k] / c.nx);
        }
    }
    volumes.assign(ng, 0);
    const double f2 = c.gb_fwhm_grid * c.gb_fwhm_grid;
    std::vector<double> gb_h((size_t)g.ncells);
    if (D == 3) {
        // labels and bisector distances on the GPU; the Gaussian on the host C library
        double* d_seeds = dalloc(seeds.size());
        int* d_vol = dalloc_t<int>(ng);
        double* d_db = gb_[0];
        const bool coloured = has_eta && c.eta_colours > 0;
        int* d_comp = coloured ? dalloc_t<int>(ns) : nullptr;
        check_cuda(cudaMemcpyAsync(d_seeds, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, stream), "H2D");
        check_cuda(cudaMemsetAsync(d_vol, 0, ng * sizeof(int), stream), "memset");
        InitParams I = init_params();
        I.ng = ng; I.nxd = c.nx; I.nyd = c.ny; I.nzd = c.nz;
        launch_voronoi3(I, d_seeds, grain, d_db, d_vol, d_comp, stream);
        std::vector<int> vol(ng);
        check_cuda(cudaMemcpyAsync(vol.data(), d_vol, ng * sizeof(int), cudaMemcpyDeviceToHost, stream), "D2H");
        copy_out(d_db, gb_h.data());
        if (coloured) {
            init_db = gb_h;
            init_comp.resize((size_t)g.ncells);
            check_cuda(cudaMemcpy2DAsync(init_comp.data(), (size_t)g.nb * sizeof(int), d_comp, (size_t)g.pb * sizeof(int),
                                         (size_t)g.nb * sizeof(int), (size_t)g.nx * g.na, cudaMemcpyDeviceToHost, stream), "D2H");
            sync();
            cudaFree(d_comp);
            dev_bytes -= ns * sizeof(int);
        }
        for (int q = 0; q < ng; ++q) volumes[q] = vol[q];
        cudaFree(d_seeds);
        cudaFree(d_vol);
        dev_bytes -= seeds.size() * 8 + ng * sizeof(int);
        parallel_for(g.ncells, [&](long long b, long long e) {
            for (long long q = b; q < e; ++q) {
                const double db = gb_h[q];
                gb_h[q] = ng == 1 ? 0. : std::exp(-4. * std::log(2.) * db * db / f2);
            }
        });
        copy_in(gb_[0], gb_h.data());
    } else {
        std::vector<double> grain_h((size_t)g.ncells);
        voronoi2d_host(grain_h, gb_h);
        copy_in(grain, grain_h.data());
        copy_in(gb_[0], gb_h.data());
    }
}

void Model::voronoi2d_host(std::vector<double>& grain_h, std::vector<double>& gb_h) {
    const int ng = (int)(seeds.size() / 2);
    const double f2 = c.gb_fwhm_grid * c.gb_fwhm_grid;
    std::vector<long long> vol(ng, 0);
    // labels first (cheap, serial for the area counts), then the mask in parallel
    std::vector<double> oy((size_t)g.ncells), rb((size_t)g.ncells);
    for (int i = 1; i <= c.nx; ++i)
        for (int j = 1; j <= c.ny; ++j) {
            const double x = i - .5, y = j - .5;
            int owner = 0;
            double rbest = std::numeric_limits<double>::infinity(), ownerY = 0.;
            for (int k = 0; k < ng; ++k) {
                const double dy = min_image(seeds[2 * k + 1] - y, c.ny);
                const double r = (seeds[2 * k] - x) * (seeds[2 * k] - x) + dy * dy;
                if (r < rbest) { rbest = r; owner = k; ownerY = y + dy; }
            }
            const size_t q = (size_t)(i - 1) * c.ny + (j - 1);
            grain_h[q] = owner + 1;
            oy[q] = ownerY;
            rb[q] = rbest;
            ++vol[owner];
        }
    parallel_for(g.ncells, [&](long long b, long long e) {
        for (long long q = b; q < e; ++q) {
            const int i = (int)(q / c.ny) + 1, j = (int)(q % c.ny) + 1;
            const double x = i - .5, y = j - .5;
            const int owner = (int)grain_h[q] - 1;
            double db = std::numeric_limits<double>::infinity();
            for (int k = 0; k < ng; ++k) {
                if (k == owner) continue;
                for (int im = -1; im <= 1; ++im) {
                    const double ym = seeds[2 * k + 1] + im * c.ny;
                    const double rs = (seeds[2 * k] - x) * (seeds[2 * k] - x) + (ym - y) * (ym - y);
                    const double sep = std::hypot(seeds[2 * k] - seeds[2 * owner], ym - oy[q]);
                    if (sep > 1.e-14) db = std::min(db, std::max(0., (rs - rb[q]) / (2. * sep)));
                }
            }
            gb_h[q] = ng == 1 ? 0. : std::exp(-4. * std::log(2.) * db * db / f2);
        }
    });
    for (int k = 0; k < ng; ++k) volumes[k] = vol[k];
}

Grid Model::own_grid() const {
    Grid o = g;
    o.nx = sp.x_hi - sp.x_lo;
    o.ncells = (long long)o.nx * g.na * g.nb;
    o.nstore = (long long)o.nx * g.plane;
    return o;
}

InitParams Model::init_params() const {
    InitParams I{};
    I.g = g;
    I.x_off = x_off;
    I.x_lo = sp.x_lo;
    I.x_hi = sp.x_hi;
    return I;
}

void Model::reset_inventory() {
    const long long off = own_offset();
    launch_diagnostics(own_grid(), o_[cur] + off, cr_[cur] + off, p_[cur] + off, diag_part, nullptr, diag_out, stream);
    DiagOut d;
    check_cuda(cudaMemcpyAsync(&d, diag_out, sizeof d, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    DevBudget b;
    check_cuda(cudaMemcpyAsync(&b, bud, sizeof b, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    b.initialO[0] = d.sum[0][0]; b.initialO[1] = d.sum[0][1];
    b.initialCr[0] = d.sum[1][0]; b.initialCr[1] = d.sum[1][1];
    check_cuda(cudaMemcpyAsync(bud, &b, sizeof b, cudaMemcpyHostToDevice, stream), "H2D");
    sync();
}

// initialize_center_oxide (3S:725-751, 2D:517-542)
void Model::init_center_seed() {
    const double x = 0.5 * (double(c.nx) + 1.), y = 0.5 * (double(c.ny) + 1.), z = 0.5 * (double(c.nz) + 1.);
    const double r = c.radius_grid;
    const int mn = dim == 3 ? std::min({c.nx, c.ny, c.nz}) : std::min(c.nx, c.ny);
    if (r >= 0.5 * (double(mn) - 1.))
        throw Error(NICR_ERR_INVALID_ARG, dim == 3 ? "Center seed is too large: --radius-grid must be less than (min(nx,ny,nz)-1)/2."
                                                   : "Center seed is too large: --radius-grid must be less than (min(nx,ny)-1)/2.");
    InitParams I = init_params();
    int nb = 0;
    launch_center_seed(I, x, y, z, r, 0, o_[cur], cr_[cur], p_[cur], nullptr, partials, stream, &nb);
    launch_reduce_partials(partials, nb, red_out, stream);
    StepPartial s;
    check_cuda(cudaMemcpyAsync(&s, red_out, sizeof s, cudaMemcpyDeviceToHost, stream), "D2H");
    DevBudget b;
    check_cuda(cudaMemcpyAsync(&b, bud, sizeof b, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    center_seed_cells = (int)s.clipped;
    // a slab may hold none of the seed; its group checks the total
    if (center_seed_cells == 0 && !is_slab) throw Error(NICR_ERR_INVALID_ARG, "Center seed covers no cell centres: increase --radius-grid.");
    b.v[0][0] = s.s[0][0]; b.v[0][1] = s.s[0][1];
    b.v[1][0] = s.s[1][0]; b.v[1][1] = s.s[1][1];
    if (x_off == 0) b.nuclei += 1;   // counted once, by the slab holding domain plane 0
    check_cuda(cudaMemcpyAsync(bud, &b, sizeof b, cudaMemcpyHostToDevice, stream), "H2D");
    sync();
}

void Model::alloc_eta(int n) {
    neta = n;
    const size_t ns = (size_t)g.nstore;
    eta_[0] = dalloc(ns * n);
    check_cuda(cudaMemsetAsync(eta_[0], 0, ns * n * 8, stream), "memset");
    if (advance_eta) eta_[1] = dalloc(ns * n);
    eta_dirty = true;
}

void Model::grain_adjacency() {
    const int ng = (int)(seeds.size() / 3);
    unsigned char* d_adj = dalloc_t<unsigned char>((size_t)ng * ng);
    check_cuda(cudaMemsetAsync(d_adj, 0, (size_t)ng * ng, stream), "memset");
    InitParams I = init_params();
    I.ng = ng;
    launch_grain_adjacency(I, grain, d_adj, stream);
    adjacency.assign((size_t)ng * ng, 0);
    check_cuda(cudaMemcpyAsync(adjacency.data(), d_adj, adjacency.size(), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    cudaFree(d_adj);
    dev_bytes -= (size_t)ng * ng;
}

std::vector<int> colour_grains(const std::vector<unsigned char>& adj, int ng, int k) {
    std::vector<int> colour((size_t)ng, -1), degree((size_t)ng, 0);
    for (int a = 0; a < ng; ++a)
        for (int b = 0; b < ng; ++b) degree[(size_t)a] += adj[(size_t)a * ng + b] != 0;
    std::vector<int> count((size_t)k);
    for (int step = 0; step < ng; ++step) {
        int v = -1, vsat = -1;
        for (int a = 0; a < ng; ++a) {
            if (colour[(size_t)a] >= 0) continue;
            std::vector<char> seen((size_t)k, 0);
            int sat = 0;
            for (int b = 0; b < ng; ++b) {
                const int cb = colour[(size_t)b];
                if (adj[(size_t)a * ng + b] && cb >= 0 && !seen[(size_t)cb]) { seen[(size_t)cb] = 1; ++sat; }
            }
            if (v < 0 || sat > vsat || (sat == vsat && degree[(size_t)a] > degree[(size_t)v])) { v = a; vsat = sat; }
        }
        std::fill(count.begin(), count.end(), 0);
        for (int b = 0; b < ng; ++b)
            if (adj[(size_t)v * ng + b] && colour[(size_t)b] >= 0) ++count[(size_t)colour[(size_t)b]];
        int best = 0;
        for (int q = 1; q < k; ++q)
            if (count[(size_t)q] < count[(size_t)best]) best = q;
        colour[(size_t)v] = best;   // the lowest free colour, else the least used among neighbours
    }
    return colour;
}

// Coloured eta (extension, eta_colours = K): every cell of grain a, whose
// nearest Voronoi bisector (distance d cells) faces grain b, gets
// eta[colour(a)] = (1 - h(phi)) (1 + tanh d) / 2 and eta[colour(b)] =
// (1 - h(phi)) (1 - tanh d) / 2: the two values meet at 1/2 on the bisector
// and the boundary is about 2 cells wide (10-90%: 2.2 cells). When a and b
// share a colour (or a is the only grain), eta[colour(a)] = 1 - h(phi).
// Every other field is 0. tanh is the host C library's.
void Model::init_eta_coloured() {
    const long long n = g.ncells;
    std::vector<double> ph((size_t)n), grain_h((size_t)n);
    copy_out(p_[cur], ph.data());
    copy_out(grain, grain_h.data());
    std::vector<double> eta_h((size_t)n * neta, 0.);
    parallel_for(n, [&](long long b, long long e) {
        for (long long q = b; q < e; ++q) {
            const int owner = int(grain_h[(size_t)q]) - 1, comp = init_comp[(size_t)q];
            const int ca = seed_colour[(size_t)owner];
            const double metal = 1. - h(ph[(size_t)q]);
            if (comp < 0 || seed_colour[(size_t)comp] == ca) {
                eta_h[(size_t)ca * n + q] = metal;
                continue;
            }
            const double t = std::tanh(init_db[(size_t)q]);
            eta_h[(size_t)ca * n + q] = metal * (0.5 * (1. + t));
            eta_h[(size_t)seed_colour[(size_t)comp] * n + q] = metal * (0.5 * (1. - t));
        }
    });
    for (int q = 0; q < neta; ++q) copy_in(eta_[0] + (size_t)q * g.nstore, eta_h.data() + (size_t)q * n);
    init_db.clear();
    init_db.shrink_to_fit();
    init_comp.clear();
    init_comp.shrink_to_fit();
    eta_dirty = true;
}

// initialize_eta (3S:469-494, 2D:293-327): weights exp(-d/ell) normalised,
// times 1-h(phi). Competitor distances on the GPU (3D), exp on the host.
void Model::init_eta() {
    const int ng = (int)(seeds.size() / dim);
    neta = ng;
    const size_t ns = (size_t)g.nstore;
    eta_[0] = dalloc(ns * ng);
    check_cuda(cudaMemsetAsync(eta_[0], 0, ns * ng * 8, stream), "memset");
    if (advance_eta) eta_[1] = dalloc(ns * ng);
    const long long n = g.ncells;
    const double ell_grid = ec.ell / c.dx;
    std::vector<double> ph((size_t)n), grain_h((size_t)n);
    copy_out(p_[cur], ph.data());
    copy_out(grain, grain_h.data());
    std::vector<double> d((size_t)n * ng);
    if (dim == 3) {
        double* d_seeds = dalloc(seeds.size());
        check_cuda(cudaMemcpyAsync(d_seeds, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, stream), "H2D");
        InitParams I = init_params();
        I.ng = ng; I.nxd = c.nx; I.nyd = c.ny; I.nzd = c.nz;
        launch_eta_dist3(I, d_seeds, grain, eta_[0], stream);
        for (int q = 0; q < ng; ++q) copy_out(eta_[0] + (size_t)q * ns, d.data() + (size_t)q * n);
        cudaFree(d_seeds);
        dev_bytes -= seeds.size() * 8;
    }
    std::vector<double> eta_h((size_t)n * ng);
    parallel_for(n, [&](long long b, long long e) {
        std::vector<double> w(ng);
        for (long long q = b; q < e; ++q) {
            const int owner = int(grain_h[q]) - 1;
            double norm = 0.;
            if (dim == 3) {
                for (int s = 0; s < ng; ++s) {
                    w[s] = s == owner ? 1. : std::exp(-d[(size_t)s * n + q] / ell_grid);
                    norm += w[s];
                }
            } else {
                const int i = (int)(q / c.ny) + 1, j = (int)(q % c.ny) + 1;
                const double x = i - .5, y = j - .5;
                const double oy = y + min_image(seeds[2 * owner + 1] - y, c.ny);
                const double rbest = std::pow(seeds[2 * owner] - x, 2) + std::pow(oy - y, 2);
                for (int s = 0; s < ng; ++s) {
                    if (s == owner) { w[s] = 1.; norm += 1.; continue; }
                    double distance = std::numeric_limits<double>::infinity();
                    for (int im = -1; im <= 1; ++im) {
                        const double gy = seeds[2 * s + 1] + im * c.ny;
                        const double sep = std::hypot(seeds[2 * s] - seeds[2 * owner], gy - oy);
                        const double rr = std::pow(seeds[2 * s] - x, 2) + std::pow(gy - y, 2);
                        if (sep > 1.e-14) distance = std::min(distance, std::max(0., (rr - rbest) / (2. * sep)));
                    }
                    w[s] = std::exp(-distance / ell_grid);
                    norm += w[s];
                }
            }
            const double metal = 1. - h(ph[q]);
            for (int s = 0; s < ng; ++s) eta_h[(size_t)s * n + q] = metal * w[s] / norm;
        }
    });
    for (int q = 0; q < ng; ++q) copy_in(eta_[0] + (size_t)q * ns, eta_h.data() + (size_t)q * n);
    eta_dirty = true;
}

void Model::eta_mask_now() {
    if (!has_eta) return;
    const size_t e = prof_begin();
    launch_eta_mask(sp, neta, eta_[ecur], gb_[gcur], s2_[gcur], dim == 2 ? pairs : nullptr, st, stream);
    prof_end(K_ETA_MASK, e, 1);
    eta_dirty = false;
}

// Ksp tables: ball and exclusion offsets, 2D hypot table (C library hypot).
void Model::setup_ksp() {
    const double r = c.radius_grid, limit = r + c.exclusion_gap_grid;
    const int rr = dim == 3 ? bounded_reach_h(r, c.nx) : int(std::ceil(r));
    const int sr = dim == 3 ? bounded_reach_h(limit, c.nx) : int(std::ceil(limit));
    const int B = rr + sr;
    std::vector<int> ball, shadow;
    if (dim == 3) {
        for (int di = -rr; di <= rr; ++di)
            for (int dj = -rr; dj <= rr; ++dj)
                for (int dk = -rr; dk <= rr; ++dk)
                    if (double(di * di) + double(dj) * dj + double(dk) * dk <= r * r) { ball.push_back(di); ball.push_back(dj); ball.push_back(dk); }
    } else {
        for (int di = -rr; di <= rr; ++di)
            for (int dj = -rr; dj <= rr; ++dj)
                if (double(di * di) + double(dj) * dj <= r * r) { ball.push_back(di); ball.push_back(dj); ball.push_back(0); }
    }
    const int nball = (int)ball.size() / 3;
    // 2D predicate table over |di| <= 2B, |dj| <= max(ny/2, 2B)
    const int hrows = 2 * B + 1, hcols = std::max(c.ny / 2 + 1, 2 * B + 1);
    std::vector<unsigned char> hyp;
    if (dim == 2) {
        hyp.resize((size_t)hrows * hcols);
        for (int a = 0; a < hrows; ++a)
            for (int b = 0; b < hcols; ++b) hyp[(size_t)a * hcols + b] = std::hypot(double(a), double(b)) < limit ? 1 : 0;
    }
    auto near = [&](int di, int dj, int dk) {
        if (dim == 3) return std::sqrt(std::pow(double(di), 2) + std::pow(double(dj), 2) + std::pow(double(dk), 2)) < limit;
        return hyp[(size_t)std::abs(di) * hcols + std::abs(dj)] != 0;
    };
    const int kz = dim == 3 ? B : 0;
    for (int di = -B; di <= B; ++di)
        for (int dj = -B; dj <= B; ++dj)
            for (int dk = -kz; dk <= kz; ++dk) {
                bool hit = false;
                for (int b = 0; b < nball && !hit; ++b)
                    hit = near(di - ball[3 * b], dj - ball[3 * b + 1], dk - ball[3 * b + 2]);
                if (hit) { shadow.push_back(di); shadow.push_back(dj); shadow.push_back(dk); }
            }
    d_ball = dalloc_t<int>(ball.size());
    d_shadow = dalloc_t<int>(shadow.size());
    check_cuda(cudaMemcpyAsync(d_ball, ball.data(), ball.size() * 4, cudaMemcpyHostToDevice, stream), "H2D");
    check_cuda(cudaMemcpyAsync(d_shadow, shadow.data(), shadow.size() * 4, cudaMemcpyHostToDevice, stream), "H2D");
    if (dim == 2) {
        d_hyp = dalloc_t<unsigned char>(hyp.size());
        check_cuda(cudaMemcpyAsync(d_hyp, hyp.data(), hyp.size(), cudaMemcpyHostToDevice, stream), "H2D");
    }
    kd.g = g;
    kd.nx = c.nx; kd.ny = c.ny; kd.nz = dim == 3 ? c.nz : 1;
    kd.radius = r; kd.gap = c.exclusion_gap_grid; kd.ksp = c.ksp;
    kd.neta = 0;  // set at scan time
    kd.hyp2d = d_hyp; kd.hyp_stride = hcols;
    kd.shadow = d_shadow; kd.n_shadow = (int)shadow.size() / 3;
    kd.ball = d_ball; kd.n_ball = nball;
    kd.full_ball = nball;
    kd.box_half = B;
    kd.x_off = x_off;
    kd.x_lo = sp.x_lo;
    kd.x_hi = sp.x_hi;
    kw.flag = dalloc_t<unsigned char>((size_t)g.ncells);
    kw.blocked = dalloc_t<unsigned char>((size_t)g.ncells);
    kw.counts = dalloc_t<int>(ksp_compact_blocks(g.ncells) + 1);
    kw.list = dalloc_t<long long>((size_t)g.ncells);
    kw.total = dalloc_t<int>(1);
    kres = dalloc_t<KspResult>(1);
    check_cuda(cudaMemsetAsync(kres, 0, sizeof(KspResult), stream), "memset");
    sync();
}

// ------------------------------------------------------------------ fields
static bool is_state_field(int f) { return f == NICR_FIELD_O || f == NICR_FIELD_CR || f == NICR_FIELD_PHI || f == NICR_FIELD_ETA; }

double* Model::state_ptr(int field, int index) {
    if (!is_state_field(field)) throw Error(NICR_ERR_INVALID_ARG, "only O, CR, PHI and ETA can be set");
    if (field == NICR_FIELD_O) return o_[cur];
    if (field == NICR_FIELD_CR) return cr_[cur];
    if (field == NICR_FIELD_PHI) return p_[cur];
    if (index < 0 || index >= neta) throw Error(NICR_ERR_INVALID_ARG, "eta index out of range");
    return eta_[ecur] + (size_t)index * g.nstore;
}

void Model::set_field(int field, int index, const double* host) {
    copy_in(state_ptr(field, index), host);
    eta_dirty = true;  // any edit invalidates the frozen-eta cache (3S:347-349)
}

void Model::copy_planes_out(const double* d, double* host, int x_begin, int count) {
    check_cuda(cudaMemcpy2DAsync(host, (size_t)g.nb * 8, d + (size_t)x_begin * g.plane, (size_t)g.pb * 8,
                                 (size_t)g.nb * 8, (size_t)count * g.na, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
}
void Model::copy_planes_in(double* d, const double* host, int x_begin, int count) {
    check_cuda(cudaMemcpy2DAsync(d + (size_t)x_begin * g.plane, (size_t)g.pb * 8, host, (size_t)g.nb * 8,
                                 (size_t)g.nb * 8, (size_t)count * g.na, cudaMemcpyHostToDevice, stream), "H2D");
    sync();
}

void Model::refresh() {
    if (has_eta && (eta_dirty || dim == 2)) eta_mask_now();
    if (!muO) {
        const size_t ns = (size_t)g.nstore;
        muO = dalloc(ns); muCr = dalloc(ns); mo = dalloc(ns); mc = dalloc(ns);
    }
    const size_t e = prof_begin();
    launch_refresh(sp, o_[cur], cr_[cur], p_[cur], gb_[gcur], muO, muCr, mo, mc, stream);
    prof_end(K_REFRESH, e, 1);
    check_cuda(cudaGetLastError(), "refresh");
}

const double* Model::field_ptr(int field, int index) {
    const double* d = nullptr;
    switch (field) {
        case NICR_FIELD_O: d = o_[cur]; break;
        case NICR_FIELD_CR: d = cr_[cur]; break;
        case NICR_FIELD_PHI: d = p_[cur]; break;
        case NICR_FIELD_ETA:
            if (index < 0 || index >= neta) throw Error(NICR_ERR_INVALID_ARG, "eta index out of range");
            d = eta_[ecur] + (size_t)index * g.nstore;
            break;
        case NICR_FIELD_MU_O: refresh(); d = muO; break;
        case NICR_FIELD_MU_CR: refresh(); d = muCr; break;
        case NICR_FIELD_M_O: refresh(); d = mo; break;
        case NICR_FIELD_M_CR: refresh(); d = mc; break;
        case NICR_FIELD_GB:
            if (has_eta && eta_dirty) eta_mask_now();
            d = gb_[gcur];
            break;
        case NICR_FIELD_GRAIN:
            if (!grain_retained) throw Error(NICR_ERR_STATE, "the initial grain map is not retained when eta evolves (3D)");
            d = grain;
            break;
        case NICR_FIELD_ETA_S2:
            if (!has_eta) throw Error(NICR_ERR_STATE, "eta_s2 exists only with evolving grains");
            if (eta_dirty) eta_mask_now();
            d = s2_[gcur];
            break;
        case NICR_FIELD_ETA_PAIRS:
            if (!has_eta || dim != 2) throw Error(NICR_ERR_STATE, "eta_pairs exists only in 2D with evolving grains");
            eta_mask_now();
            d = pairs;
            break;
        case NICR_FIELD_GB_INITIAL:
            if (dim != 2) throw Error(NICR_ERR_STATE, "gb_initial exists only in 2D");
            d = gb_initial;
            break;
        default: throw Error(NICR_ERR_INVALID_ARG, "unknown field");
    }
    return d;
}

void Model::get_field(int field, int index, double* host) { copy_out(field_ptr(field, index), host); }

// ------------------------------------------------------------------ stepping
void Model::reset_status() {
    // keep steps_done; clear the failure state for a new batch
    h_st->err_key = ERR_NONE;
    h_st->failed = 0;
    h_st->timeout = 0;
    h_st->failed_step = -1;
    h_st->steps_done = steps_done;
    h_st->slot_err[0] = h_st->slot_err[1] = ERR_NONE;
    check_cuda(cudaMemcpyAsync(st, h_st, sizeof(Status), cudaMemcpyHostToDevice, stream), "H2D");
}

void Model::set_xchunk(int c) {
    sync();
    sp.xchunk = std::max(1, std::min(c, g.nx));
    const int need = std::max(step_main_blocks(sp), 148 * 4) + 8;
    if (need > partial_cap) {
        cudaFree(partials);
        partials = nullptr;
        partial_cap = need;
        partials = dalloc_t<StepPartial>(partial_cap);
    }
    for (auto& q : pair_graphs)   // captured launches carry the old grid
        if (q.exec) { cudaGraphExecDestroy(q.exec); q.exec = nullptr; }
}

void Model::launch_trial_eta() {
    if (advance_eta)
        launch_eta_update(sp, neta, eta_[ecur], s2_[gcur], p_[cur], eta_[ecur ^ 1], gb_[gcur ^ 1], s2_[gcur ^ 1], st,
                          stream);
}

void Model::launch_trial_kernels() {
    int nb = 0;
    if (onepass_step() && launch_onepass(&nb)) return;
    const BatchDomain d = step_desc();
    launch_step_main(sp, d.o, d.cr, d.p, d.gb, d.s2, d.on, d.crn, d.pn, partials, st, stream, &nb);
    launch_trial_eta();
}

void Model::tune(int reps, int* xchunk, int* minb) {
    reps = std::max(1, reps);
    if (!onepass_step()) prepare_step();
    reset_status();   // trial kernels of a failing state must not stop the timing runs
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    int best_c = sp.xchunk, best_m = sp.minb;
    float best_ms = -1.f;
    const std::vector<int> minbs = dim == 3 ? std::vector<int>{2, 3} : std::vector<int>{0};
    for (int c : xchunk_candidates(g.nx)) {
        set_xchunk(c);
        for (int mb : minbs) {
            sp.minb = mb;
            step_kernels_prepare(sp);
            if (onepass_step()) step_fused_prepare(sp, neta);
            launch_trial_kernels();   // warm-up
            check_cuda(cudaEventRecord(e0, stream), "cudaEventRecord");
            for (int r = 0; r < reps; ++r) launch_trial_kernels();
            check_cuda(cudaEventRecord(e1, stream), "cudaEventRecord");
            check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (best_ms < 0.f || ms < best_ms) { best_ms = ms; best_c = c; best_m = mb; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_cuda(cudaGetLastError(), "tune");
    set_xchunk(best_c);   // also drops captured step graphs
    sp.minb = best_m;
    reset_status();
    sync();
    if (xchunk) *xchunk = best_c;
    if (minb) *minb = best_m;
}

void Model::prepare_step() {
    if (has_eta && eta_dirty) eta_mask_now();
}

BatchDomain Model::step_desc() const {
    BatchDomain d{};
    const int nxt = cur ^ 1;
    d.sp = sp;
    d.o = o_[cur]; d.cr = cr_[cur]; d.p = p_[cur];
    d.gb = gb_[gcur];
    d.s2 = has_eta ? s2_[gcur] : nullptr;
    d.on = o_[nxt]; d.crn = cr_[nxt]; d.pn = p_[nxt];
    d.partials = partials;
    d.st = st;
    return d;
}

FinalizeDomain Model::finalize_desc(int nb) const {
    FinalizeDomain f{};
    f.partials = partials;
    f.nblocks = nb;
    f.budget = bud;
    f.st = st;
    return f;
}

void Model::complete_step(int nb, bool finalize) {
    if (advance_eta) {
        const size_t e = prof_begin();
        launch_eta_update(sp, neta, eta_[ecur], s2_[gcur], p_[cur], eta_[ecur ^ 1], gb_[gcur ^ 1], s2_[gcur ^ 1], st, stream);
        prof_end(K_ETA_UPDATE, e, 1);
    }
    if (finalize) {
        const size_t e = prof_begin();
        launch_step_finalize(partials, nb, bud, st, 0, stream);
        prof_end(K_FINALIZE, e, 1);
    }
    cur ^= 1;
    if (advance_eta) { ecur ^= 1; gcur ^= 1; }
}

bool Model::fused_step() const {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NICR_FUSED");
        v = (e && e[0] == '1') ? 1 : 0;
    }
    return v == 1 && sp.fast && dim == 3 && advance_eta && !is_slab && neta >= 1 && neta <= 16;
}

bool Model::onepass_step() const {
    static int env = -1;   // NICR_STEP_FORM: 1 onepass, 2 split, 0 unset
    if (env < 0) {
        const char* e = getenv("NICR_STEP_FORM");
        env = (e && e[0] == 'o') ? NICR_STEP_ONEPASS : (e && e[0] == 's') ? NICR_STEP_SPLIT : 0;
    }
    const int form = env ? env : c.step_form;
    const bool want = form != NICR_STEP_SPLIT;
    return want && !onepass_failed && dim == 3 && advance_eta && !is_slab && !fused_step() &&
           step_fused_applies(g, neta);
}

bool Model::launch_onepass(int* nb) {
    const size_t e = prof_begin();
    if (!launch_step_fused(sp, neta, o_[cur], cr_[cur], p_[cur], eta_[ecur], o_[cur ^ 1], cr_[cur ^ 1], p_[cur ^ 1],
                           eta_[ecur ^ 1], partials, st, stream, nb)) {
        onepass_failed = true;
        return false;
    }
    prof_end(K_STEP_FUSED, e, 1);
    return true;
}

void Model::enqueue_step() {
    int nb = 0;
    if (onepass_step()) {
        if (launch_onepass(&nb)) {
            const size_t e = prof_begin();
            launch_step_finalize(partials, nb, bud, st, 0, stream);
            prof_end(K_FINALIZE, e, 1);
            cur ^= 1;
            ecur ^= 1;
            gcur ^= 1;
            eta_dirty = true;   // gb and eta_s2 were not written: rebuilt from eta when read
            return;
        }
    }
    prepare_step();
    const BatchDomain d = step_desc();
    if (fused_step()) {
        if (!ticket) ticket = dalloc_t<unsigned>(1);
        size_t e = prof_begin();
        launch_step_eta_fast(sp, neta, d.o, d.cr, d.p, d.gb, d.s2, d.on, d.crn, d.pn, partials, eta_[ecur],
                             eta_[ecur ^ 1], gb_[gcur ^ 1], s2_[gcur ^ 1], ticket, st, stream, &nb);
        prof_end(K_STEP_ETA, e, 1);
        e = prof_begin();
        launch_step_finalize(partials, nb, bud, st, 0, stream);
        prof_end(K_FINALIZE, e, 1);
        cur ^= 1;
        ecur ^= 1;
        gcur ^= 1;
        return;
    }
    const size_t e = prof_begin();
    launch_step_main(sp, d.o, d.cr, d.p, d.gb, d.s2, d.on, d.crn, d.pn, partials, st, stream, &nb);
    prof_end(K_STEP_MAIN, e, step_main_kernels(sp));
    complete_step(nb, true);
}

std::string Model::describe_failure(unsigned long long key, int nxt) {
    std::ostringstream msg;
    auto coords = [&](long long cell, int& i, int& j, int& k) {
        const int col = (int)(cell % g.nb);
        const long long r = cell / g.nb;
        const int row = (int)(r % g.na);
        i = (int)(r / g.na) + 1;
        if (dim == 3) { j = row + 1; k = col + 1; } else { j = col + 1; k = 0; }
        return (long long)(i - 1 - x_off) * g.plane + (long long)row * g.pb + col;
    };
    // a slab describes only failures in its own planes (its group asks the owner)
    auto owned = [&](long long cell) {
        const long long xi = cell / ((long long)g.na * g.nb) - x_off;
        return xi >= sp.x_lo && xi < sp.x_hi;
    };
    int i, j, k;
    if (key < ERR_ETA_BASE) {
        const long long cell = (long long)(key / 4);
        if (!owned(cell)) return std::string();
        if (key % 4 == 0) return "Nonfinite trial field: reduce dt / inspect the model; no update accepted.";
        const long long idx = coords(cell, i, j, k);
        double v[3];
        check_cuda(cudaMemcpyAsync(&v[0], o_[nxt] + idx, 8, cudaMemcpyDeviceToHost, stream), "D2H");
        check_cuda(cudaMemcpyAsync(&v[1], cr_[nxt] + idx, 8, cudaMemcpyDeviceToHost, stream), "D2H");
        check_cuda(cudaMemcpyAsync(&v[2], p_[nxt] + idx, 8, cudaMemcpyDeviceToHost, stream), "D2H");
        sync();
        msg << std::scientific << std::setprecision(16) << "Out-of-bounds trial at (" << i << "," << j;
        if (dim == 3) msg << "," << k;
        msg << "): O=" << v[0] << ", Cr=" << v[1] << ", phi=" << v[2]
            << ". No clipping/update accepted. Reduce dt; if failure persists, investigate model.";
        return msg.str();
    }
    const unsigned long long q = key - ERR_ETA_BASE;
    const int gi = (int)(q / (unsigned long long)sp.key_ncells);
    if (!owned((long long)(q % (unsigned long long)sp.key_ncells))) return std::string();
    const long long idx = coords((long long)(q % (unsigned long long)sp.key_ncells), i, j, k);
    double v;
    check_cuda(cudaMemcpyAsync(&v, eta_[ecur ^ 1] + (size_t)gi * g.nstore + idx, 8, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    msg << std::setprecision(17) << "Eta trial outside [0,1]: grain=" << gi + 1 << " cell=(" << i << "," << j;
    if (dim == 3) msg << "," << k;
    msg << ") value=" << v << ". All PDE fields rejected together; eta is never clipped. Check eta coefficients/dt.";
    return msg.str();
}

int Model::finish_batch(long long before, int enqueued, const std::vector<double>* nuc_sched, int* completed) {
    check_cuda(cudaMemcpyAsync(h_st, st, sizeof(Status), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_cuda(cudaGetLastError(), "step kernels");
    profile_collect();
    if (h_st->timeout)
        throw Error(NICR_ERR_CUDA, "a step kernel's bounded wait for its own copies ran out; the step results are not valid");
    if (!h_st->failed) {
        steps_done = before + enqueued;
        if (completed) *completed = enqueued;
        return NICR_OK;
    }
    const int accepted = (int)(h_st->failed_step - before);
    // every step toggled the buffer parity; the valid state is the input of the failed step
    const int undo = (enqueued - accepted) & 1;
    cur ^= undo;
    if (advance_eta) { ecur ^= undo; gcur ^= undo; }
    steps_done = before + accepted;
    if (completed) *completed = accepted;
    if (nuc_sched) next_nucleation = (*nuc_sched)[accepted];
    const unsigned long long key = h_st->err_key;
    last_error = describe_failure(key, cur ^ 1);
    if (dim == 2 && sp.inlet) {
        // 2D leaves the enforced inlet layer in place after a rejection (2D:553, 2D:1224)
        std::vector<double> plane((size_t)g.nb, c.layer_o);
        check_cuda(cudaMemcpyAsync(o_[cur], plane.data(), plane.size() * 8, cudaMemcpyHostToDevice, stream), "H2D");
        sync();
        // the enforce_legacy_layer increment is part of the rolled-back budget
    }
    if (has_eta) eta_dirty = true;
    if (key < ERR_ETA_BASE) return key % 4 == 0 ? NICR_ERR_TRIAL_NONFINITE : NICR_ERR_TRIAL_BOUNDS;
    return NICR_ERR_ETA_RANGE;
}

void Model::run_begin(RunPlan& r, int nsteps, bool schedule) {
    reset_status();
    r.before = steps_done;
    r.nsteps = nsteps;
    r.schedule = schedule;
    r.next = next_nucleation;
    r.sched.assign(schedule ? (size_t)nsteps + 1 : 0, 0.);
}

void Model::run_pre_step(RunPlan& r, int s) {
    if (!r.schedule) return;
    const long long n = r.before + s + 1;
    const double time = double(n) * c.dt;
    if (c.nucleation == NICR_NUC_KSP && time + 1.e-12 * c.nucleation_period >= r.next) {
        kd.neta = neta;
        const size_t e = prof_begin();
        launch_ksp_scan(kd, o_[cur], cr_[cur], p_[cur], eta_[ecur], kw, bud, kres, st, stream);
        prof_end(K_KSP, e, 4);
        if (has_eta) eta_dirty = true;
        r.next += c.nucleation_period;
    }
    r.sched[(size_t)s] = r.next;
}

int Model::run_end(RunPlan& r, int* completed) {
    if (!r.schedule) return finish_batch(r.before, r.nsteps, nullptr, completed);
    r.sched[(size_t)r.nsteps] = r.next;
    const int rc = finish_batch(r.before, r.nsteps, &r.sched, completed);
    if (rc == NICR_OK) next_nucleation = r.next;
    return rc;
}

bool Model::ksp_due(const RunPlan& r, int s) const {
    if (!r.schedule || c.nucleation != NICR_NUC_KSP) return false;
    const long long n = r.before + s + 1;
    return double(n) * c.dt + 1.e-12 * c.nucleation_period >= r.next;
}

// Step graphs. Replaying a captured run of 2..16 steps costs one host launch
// instead of two or three per step, which decides the step rate of small
// domains (a 2D 128^2 step is a few microseconds of GPU work). An even run
// returns the buffer parity to where it started, so one graph per length and
// starting parity serves every run; the kernels read their run constants from their
// parameters and the batch-stop flag from device memory, both unchanged
// between replays. Not used while profiling (the per-kernel events) or when
// NICR_GRAPHS=0.
bool Model::graphs_enabled() const {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("NICR_GRAPHS");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1 && !prof_on;
}

void Model::launch_step_group(int n) {
    if (!onepass_step()) prepare_step();   // a stale eta mask is rebuilt outside the graph
    const int key = cur | (ecur << 1) | (gcur << 2) | (n << 3);
    PairGraph* pg = nullptr;
    for (auto& q : pair_graphs)
        if (q.exec && q.key == key) pg = &q;
    if (!pg) {
        for (auto& q : pair_graphs)
            if (!q.exec) { pg = &q; break; }
        if (!pg) throw Error(NICR_ERR_STATE, "step graph slots exhausted");
        step_kernels_prepare(sp);
        if (onepass_step()) step_fused_prepare(sp, neta);   // kernel attributes outside the capture
        if (fused_step()) {
            if (!ticket) ticket = dalloc_t<unsigned>(1);
            step_eta_prepare_fast(sp, neta);   // kernel attributes outside the capture
        }
        const long long l0 = launches;
        cudaGraph_t graph = nullptr;
        check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        for (int q = 0; q < n; ++q) enqueue_step();
        check_cuda(cudaStreamEndCapture(stream, &graph), "cudaStreamEndCapture");
        const cudaError_t e = cudaGraphInstantiate(&pg->exec, graph, 0);
        cudaGraphDestroy(graph);
        check_cuda(e, "cudaGraphInstantiate");
        pg->key = key;
        pg->kernels = launches - l0;
        launches = l0;   // nothing ran while capturing; each replay counts them
        // the captured enqueue_step calls toggled the parity an even number of times: back at key
    }
    check_cuda(cudaGraphLaunch(pg->exec, stream), "cudaGraphLaunch");
    launches += pg->kernels;
}

// The longest captured run (16, 8, 4 or 2 steps) that starts at step s of
// plan r, fits in the batch and has no Ksp scan due after its first step;
// 1 when none does (a plain launch).
int Model::group_length(const RunPlan& r, int s, int nsteps) const {
    for (int g : {16, 8, 4, 2}) {
        if (s + g > nsteps) continue;
        bool ok = true;
        for (int j = 1; j < g && ok; ++j) ok = !ksp_due(r, s + j);
        if (ok) return g;
    }
    return 1;
}

int Model::step(int nsteps, int* completed) {
    if (is_slab) throw Error(NICR_ERR_STATE, "a slab is advanced by its slab group");
    if (completed) *completed = 0;
    if (nsteps <= 0) return NICR_OK;
    RunPlan r;
    run_begin(r, nsteps, false);
    const bool graphs = graphs_enabled();
    for (int s = 0; s < nsteps;) {
        const int g = graphs ? group_length(r, s, nsteps) : 1;
        if (g > 1) launch_step_group(g);
        else enqueue_step();
        s += g;
    }
    return run_end(r, completed);
}

int Model::run(int nsteps, int* completed) {
    if (is_slab) throw Error(NICR_ERR_STATE, "a slab is advanced by its slab group");
    if (completed) *completed = 0;
    if (nsteps <= 0) return NICR_OK;
    RunPlan r;
    run_begin(r, nsteps, true);
    const bool graphs = graphs_enabled();
    for (int s = 0; s < nsteps;) {
        run_pre_step(r, s);
        const int g = graphs ? group_length(r, s, nsteps) : 1;
        if (g > 1) launch_step_group(g);
        else enqueue_step();
        for (int j = 1; j < g; ++j) run_pre_step(r, s + j);   // no scan is due: schedule entries only
        s += g;
    }
    return run_end(r, completed);
}

int Model::slab_launch() {
    prepare_step();
    StepParams P = sp;
    P.err_slot = cur;   // one error word per buffer parity: consecutive steps alternate
    int nb = 0;
    size_t e = prof_begin();
    launch_step_main(P, o_[cur], cr_[cur], p_[cur], gb_[gcur], has_eta ? s2_[gcur] : nullptr, o_[cur ^ 1],
                     cr_[cur ^ 1], p_[cur ^ 1], partials, st, stream, &nb);
    prof_end(K_STEP_MAIN, e, step_main_kernels(P));
    if (advance_eta) {
        e = prof_begin();
        launch_eta_update(P, neta, eta_[ecur], s2_[gcur], p_[cur], eta_[ecur ^ 1], gb_[gcur ^ 1], s2_[gcur ^ 1], st, stream);
        prof_end(K_ETA_UPDATE, e, 1);
    }
    return nb;
}

void Model::slab_commit(int nblocks, const SlabPeers& peers) {
    SlabPeers q = peers;
    q.slot = cur;
    const size_t e = prof_begin();
    launch_step_finalize_slab(partials, nblocks, bud, st, q, stream);
    prof_end(K_FINALIZE, e, 1);
    cur ^= 1;
    if (advance_eta) { ecur ^= 1; gcur ^= 1; }
}

long long* Model::d_agree() {
    if (!agree) agree = dalloc_t<long long>(1);
    return agree;
}

void Model::rank_launch() {
    const int parity = cur;
    rank_nb = slab_launch();
    launch_agree_word(st, parity, d_agree(), stream);
    launches += 1;
}

void Model::rank_commit() {
    const size_t e = prof_begin();
    launch_step_finalize_agreed(partials, rank_nb, bud, st, d_agree(), stream);
    prof_end(K_FINALIZE, e, 1);
    cur ^= 1;
    if (advance_eta) { ecur ^= 1; gcur ^= 1; }
}

void Model::adopt_stream(cudaStream_t s) {
    sync();
    if (stream && owns_stream) cudaStreamDestroy(stream);
    stream = s;
    owns_stream = false;
}

int Model::nucleate(int* nuclei) {
    if (nuclei) *nuclei = 0;
    if (c.nucleation != NICR_NUC_KSP) return NICR_OK;
    reset_status();
    kd.neta = neta;
    launch_ksp_scan(kd, o_[cur], cr_[cur], p_[cur], eta_[ecur], kw, bud, kres, st, stream);
    KspResult r;
    check_cuda(cudaMemcpyAsync(&r, kres, sizeof r, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_cuda(cudaGetLastError(), "ksp");
    if (has_eta && r.nuclei) eta_dirty = true;
    if (nuclei) *nuclei = r.nuclei;
    return NICR_OK;
}

int Model::stamp(int x, int y, int z, int* cells) {
    if (cells) *cells = 0;
    if (x < 1 || x > c.nx || y < 1 || y > c.ny || (dim == 3 && (z < 1 || z > c.nz)))
        throw Error(NICR_ERR_INVALID_ARG, "stamp centre outside the grid");
    if (!kres) {
        // stamps outside Ksp mode need the ball tables too
        setup_ksp();
    }
    reset_status();
    kd.neta = neta;
    launch_ksp_stamp(kd, x, y, dim == 3 ? z : 0, o_[cur], cr_[cur], p_[cur], eta_[ecur], kw, bud, kres, st, stream);
    KspResult r;
    check_cuda(cudaMemcpyAsync(&r, kres, sizeof r, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_cuda(cudaGetLastError(), "stamp");
    if (has_eta && r.last_cells) eta_dirty = true;
    if (cells) *cells = r.last_cells;
    return NICR_OK;
}

void Model::budget(nicr_budget* out) {
    DevBudget b;
    check_cuda(cudaMemcpyAsync(&b, bud, sizeof b, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    double* dst[8] = {out->nucO, out->nucCr, out->ckO, out->ckCr, out->clipO, out->clipCr, out->bcO, out->bcCr};
    for (int q = 0; q < 8; ++q) { dst[q][0] = b.v[q][0]; dst[q][1] = b.v[q][1]; }
    out->nuclei = b.nuclei;
    out->clipped = b.clipped;
    out->initialO[0] = b.initialO[0]; out->initialO[1] = b.initialO[1];
    out->initialCr[0] = b.initialCr[0]; out->initialCr[1] = b.initialCr[1];
}

void Model::diagnostics(nicr_diagnostics* d) {
    const long long off = own_offset();
    launch_diagnostics(own_grid(), o_[cur] + off, cr_[cur] + off, p_[cur] + off, diag_part, nullptr, diag_out, stream);
    DiagOut r;
    check_cuda(cudaMemcpyAsync(&r, diag_out, sizeof r, cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_cuda(cudaGetLastError(), "diagnostics");
    d->sum_O[0] = r.sum[0][0]; d->sum_O[1] = r.sum[0][1];
    d->sum_Cr[0] = r.sum[1][0]; d->sum_Cr[1] = r.sum[1][1];
    d->sum_phi[0] = r.sum[2][0]; d->sum_phi[1] = r.sum[2][1];
    d->sum_h[0] = r.sum[3][0]; d->sum_h[1] = r.sum[3][1];
    d->min_O = r.mn[0]; d->max_O = r.mx[0];
    d->min_Cr = r.mn[1]; d->max_Cr = r.mx[1];
    d->min_Ni = r.mn[2];
    d->min_phi = r.mn[3]; d->max_phi = r.mx[3];
}

// grain_log values (3S:566-590, 2D:382-406)
void Model::grain_stats(nicr_grain_stats* out, long long* cells, double* amount) {
    if (!has_eta) throw Error(NICR_ERR_STATE, "grain statistics exist only with evolving grains");
    if (eta_dirty || dim == 2) eta_mask_now();
    if (!gw.cells) {
        gw.cells = dalloc_t<unsigned long long>((size_t)neta);
        gw.parts = dalloc_t<unsigned char>((size_t)grain_blocks(g.ncells) * grain_part_bytes());
        gw.amount_parts = dalloc((size_t)grain_blocks(g.ncells) * neta * 2);
        g_out = dalloc_t<GrainOut>(1);
        g_amount = dalloc((size_t)neta * 2);
        g_cells = dalloc_t<long long>((size_t)neta);
    }
    // the own planes (a whole domain: all); eta fields keep their stored stride
    GrainParams G{};
    G.g = own_grid();
    G.g.nstore = g.nstore;
    G.dim = dim; G.neta = neta;
    G.dx = c.dx; G.da = c.dy; G.db = dim == 3 ? c.dz : c.dy;
    G.K = ec.K; G.W = c.eta_W; G.A = ec.A;
    G.pairs = pairs;
    G.x_above = x_off + sp.x_hi < c.nx ? 1 : 0;
    const long long off = own_offset();
    launch_grain_stats(G, eta_[ecur] + off, s2_[gcur] + off, p_[cur] + off, gb_[gcur] + off, gw, g_out, g_amount,
                       g_cells, stream);
    GrainOut r;
    check_cuda(cudaMemcpyAsync(&r, g_out, sizeof r, cudaMemcpyDeviceToHost, stream), "D2H");
    if (cells) check_cuda(cudaMemcpyAsync(cells, g_cells, (size_t)neta * sizeof(long long), cudaMemcpyDeviceToHost, stream), "D2H");
    if (amount) check_cuda(cudaMemcpyAsync(amount, g_amount, (size_t)neta * 2 * sizeof(double), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_cuda(cudaGetLastError(), "grain statistics");
    out->min_eta = r.lo; out->max_eta = r.hi; out->min_s2 = r.slo; out->max_s2 = r.shi;
    out->sum_s2[0] = r.sum[0][0]; out->sum_s2[1] = r.sum[0][1];
    out->mask[0] = r.sum[1][0]; out->mask[1] = r.sum[1][1];
    out->energy[0] = r.sum[2][0]; out->energy[1] = r.sum[2][1];
    out->gb_max = r.gbmax;
    out->unassigned = r.unassigned;
    long long alive = 0;
    std::vector<long long> cc((size_t)neta);
    check_cuda(cudaMemcpy(cc.data(), g_cells, (size_t)neta * sizeof(long long), cudaMemcpyDeviceToHost), "D2H");
    for (long long v : cc) alive += v > 0;
    out->alive = alive;
}

// ------------------------------------------------------------------ measurement hooks
const char* Model::kernel_name(int k) {
    static const char* names[K_COUNT] = {"step_main", "eta_update", "step_finalize", "eta_mask", "ksp_scan",
                                         "refresh", "diagnostics", "step_eta", "step_fused"};
    return (k >= 0 && k < K_COUNT) ? names[k] : "?";
}

void Model::profile_enable(bool on) {
    sync();
    prof_on = on;
    prof_used = 0;
    prof_marks.clear();
    for (int k = 0; k < K_COUNT; ++k) { prof_ms[k] = 0.; prof_n[k] = 0; }
}

size_t Model::prof_begin() {
    if (!prof_on) return 0;
    if (prof_used + 2 > prof_pool.size()) {
        for (int q = 0; q < 64; ++q) {
            cudaEvent_t e;
            check_cuda(cudaEventCreate(&e), "cudaEventCreate");
            prof_pool.push_back(e);
        }
    }
    const size_t e0 = prof_used;
    prof_used += 2;
    check_cuda(cudaEventRecord(prof_pool[e0], stream), "cudaEventRecord");
    return e0;
}

void Model::prof_end(int k, size_t e0, int kernels) {
    launches += kernels;
    if (!prof_on) return;
    check_cuda(cudaEventRecord(prof_pool[e0 + 1], stream), "cudaEventRecord");
    prof_marks.push_back(Mark{k, e0});
}

void Model::profile_collect() {
    if (!prof_on) return;
    sync();
    for (const Mark& m : prof_marks) {
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, prof_pool[m.e0], prof_pool[m.e0 + 1]), "cudaEventElapsedTime");
        prof_ms[m.k] += ms;
        prof_n[m.k] += 1;
    }
    prof_marks.clear();
    prof_used = 0;
}

}  // namespace nicr
