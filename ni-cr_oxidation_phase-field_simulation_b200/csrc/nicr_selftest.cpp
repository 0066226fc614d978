// --self-test: the reference's built-in verification (3S:1102-1251,
// 2D:792-931 and 2D:1011-1106) re-expressed against the GPU model. Each check
// names the reference requirement it mirrors; failures print the reference's
// "Self-test failed: ..." message.
#include <algorithm>
#include <array>
#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_model.h"

namespace {

using nicr::Model;

void require(bool v, const char* msg) {
    if (!v) throw std::runtime_error(std::string("Self-test failed: ") + msg);
}
bool near(long double a, long double b, long double atol = 1.e-11L, long double rtol = 1.e-11L) {
    return std::fabs(a - b) <= atol + rtol * std::max(std::fabs(a), std::fabs(b));
}
long double ld(const double v[2]) { return (long double)v[0] + (long double)v[1]; }

nicr_config base(int dim) {
    nicr_config c;
    nicr_config_default(&c, dim);
    if (dim == 3) { c.nx = 23; c.ny = 13; c.nz = 11; c.grain_diameter_grid = 12.; }
    else { c.nx = 31; c.ny = 25; c.grain_diameter_grid = 10.; }
    c.bc = NICR_BC_CLOSED; c.ck = NICR_CK_OFF; c.nucleation = NICR_NUC_OFF; c.dt = 1.e-12; c.radius_grid = 2.5;
    return c;
}

std::vector<double> get(Model& m, int f, int idx = 0) {
    std::vector<double> v((size_t)m.g.ncells);
    m.get_field(f, idx, v.data());
    return v;
}
long double total(Model& m, int f) {
    long double s = 0;
    for (double x : get(m, f)) s += x;
    return s;
}
// smooth fields (fill_smooth, 3S:1092-1101)
void fill_smooth(Model& m) {
    const auto& c = m.c;
    const long long n = m.g.ncells;
    std::vector<double> o((size_t)n), cr((size_t)n), p((size_t)n);
    std::vector<std::vector<double>> eta((size_t)m.neta, std::vector<double>((size_t)n));
    long long q = 0;
    const int nz = m.dim == 3 ? c.nz : 1;
    for (int i = 1; i <= c.nx; ++i)
        for (int j = 1; j <= c.ny; ++j)
            for (int k = 1; k <= nz; ++k, ++q) {
                o[q] = .001 * (1. + .08 * std::sin(.3 * i + .5 * j - .4 * k));
                cr[q] = .19 + .001 * std::cos(.2 * i - .3 * j + .6 * k);
                p[q] = .1 + .01 * std::cos(.1 * i + .4 * j - .2 * k);
                for (int g = 0; g < m.neta; ++g) eta[g][q] = .2 + .02 * std::cos(.2 * i - .3 * j + .7 * g + .5 * k);
            }
    m.set_field(NICR_FIELD_O, 0, o.data());
    m.set_field(NICR_FIELD_CR, 0, cr.data());
    m.set_field(NICR_FIELD_PHI, 0, p.data());
    for (int g = 0; g < m.neta; ++g) m.set_field(NICR_FIELD_ETA, g, eta[g].data());
}
void step(Model& m, int n = 1) {
    int done = 0;
    const int rc = m.step(n, &done);
    if (rc != NICR_OK) throw std::runtime_error(m.last_error);
}

void test_geometry(int dim) {
    nicr_config c = base(dim);
    Model s(c), repeat(c);
    require(get(s, NICR_FIELD_GRAIN) == get(repeat, NICR_FIELD_GRAIN) && get(s, NICR_FIELD_GB) == get(repeat, NICR_FIELD_GB),
            "seed reproducibility");
    const double vol = dim == 3 ? double(c.nx) * c.ny * c.nz : double(c.nx) * c.ny;
    const int ng = dim == 3 ? std::max(1, int(std::llround(6. * vol / (nicr::PI * std::pow(c.grain_diameter_grid, 3)))))
                            : std::max(1, int(std::llround(4. * vol / (nicr::PI * c.grain_diameter_grid * c.grain_diameter_grid))));
    require((int)s.volumes.size() == ng, "volume-based grain count");
    long long count = 0;
    for (long long v : s.volumes) count += v;
    require(count == (long long)vol, "grain volumes cover box");
    for (double g : get(s, NICR_FIELD_GB)) require(g >= 0. && g <= 1., "bounded fixed GB mask");
    for (double g : get(s, NICR_FIELD_GRAIN)) require(g >= 1., "complete Voronoi coverage");
    nicr_config changed = c;
    ++changed.random_seed;
    Model other(changed);
    require(get(other, NICR_FIELD_GRAIN) != get(s, NICR_FIELD_GRAIN), "different seed changes geometry");
    if (dim == 3) {
        const auto g = get(s, NICR_FIELD_GRAIN);
        bool differs = false;
        for (long long q = 0; q < s.g.ncells; ++q) differs = differs || g[q] != g[q - q % c.nz];
        require(differs, "3D grains are not an extruded 2D map");
    }
    // anchored inlet sites own inlet-face cells (3S:1134-1138, 2D:793-801)
    for (int seed = 0; seed < 4; ++seed) {
        nicr_config t = c;
        t.random_seed = seed;
        t.left_edge_sites = dim == 3 ? ng : std::min(ng, 2);
        Model m(t);
        const auto g = get(m, NICR_FIELD_GRAIN);
        std::vector<bool> seen(t.left_edge_sites, false);
        const long long face = dim == 3 ? (long long)c.ny * c.nz : c.ny;
        for (long long q = 0; q < face; ++q) {
            const int id = int(g[q]) - 1;
            if (id < t.left_edge_sites) seen[id] = true;
        }
        for (bool v : seen) require(v, "anchored sites each own inlet-face cells");
    }
    nicr_config t = c;
    t.grains = 0;
    Model single(t);
    require(single.volumes[0] == (long long)vol && total(single, NICR_FIELD_GB) == 0., "single-crystal volume and mask");
    t = c;
    t.grain_diameter_grid = 10000.;
    Model one(t);
    require(total(one, NICR_FIELD_GB) == 0., "own periodic images do not make a GB");
    t = c;
    t.left_edge_sites = ng + 1;
    bool rejected = false;
    try { Model bad(t); } catch (const std::exception&) { rejected = true; }
    require(rejected, "excess anchors rejected");
    std::cout << "PASS: " << dim << "D Voronoi volume rule, coverage, reproducibility, inlet anchors and limits.\n";
}

void test_transport(int dim) {
    nicr_config c = base(dim);
    Model s(c);
    fill_smooth(s);
    const long double so = total(s, NICR_FIELD_O), sc = total(s, NICR_FIELD_CR);
    step(s);
    require(near(total(s, NICR_FIELD_O), so) && near(total(s, NICR_FIELD_CR), sc), "closed transport conserves O and Cr");
    const double gbf_o = nicr::mobility(.1, 0., 1., nicr::Phys::bmo, nicr::Phys::boo, c.gb_factor_o - 1.) /
                         nicr::mobility(.1, 0., 0., nicr::Phys::bmo, nicr::Phys::boo, c.gb_factor_o - 1.);
    require(near(gbf_o, c.gb_factor_o), "O GB mobility factor");
    for (int bc : {NICR_BC_MU, NICR_BC_CLOSED, NICR_BC_CONCENTRATION}) {
        nicr_config t = c;
        t.bc = bc;
        t.oxygen_diffusion = 0;
        Model m(t);
        fill_smooth(m);
        const auto old = get(m, NICR_FIELD_O);
        step(m, 3);
        nicr_budget b;
        m.budget(&b);
        require(get(m, NICR_FIELD_O) == old && ld(b.bcO) == 0., "O off freezes O transport/inlet on every BC");
    }
    nicr_config t = c;
    t.bc = NICR_BC_MU;
    Model dry(t);
    step(dry);
    nicr_budget b;
    dry.budget(&b);
    require(total(dry, NICR_FIELD_O) > 0. && near(total(dry, NICR_FIELD_O) - ld(b.initialO), ld(b.bcO)), "mu inlet face inventory balance");
    t.bc = NICR_BC_CONCENTRATION;
    Model layer(t);
    step(layer);
    layer.budget(&b);
    require(near(total(layer, NICR_FIELD_O) - ld(b.initialO), ld(b.bcO)), "concentration inlet inventory balance");
    require(std::fabs((12000000. * .0023 + 3200000. * .1986 - 298432.) - 364688.) < 1.e-8, "mu reference arithmetic");
    std::cout << "PASS: " << dim << "D conservative flux, O/Cr budgets, mobility gates and oxygen switch.\n";
}

void test_seeds(int dim) {
    nicr_config c = base(dim);
    const std::vector<std::array<int, 3>> boxes = dim == 3 ? std::vector<std::array<int, 3>>{{17, 15, 13}, {18, 16, 14}}
                                                           : std::vector<std::array<int, 3>>{{31, 25, 1}, {32, 26, 1}};
    for (const auto& bx : boxes) {
        nicr_config t = c;
        t.nx = bx[0]; t.ny = bx[1]; t.nz = bx[2];
        t.grains = 0; t.nucleation = NICR_NUC_CENTER; t.radius_grid = 3.5;
        Model m(t);
        const auto p = get(m, NICR_FIELD_PHI);
        const double cx = .5 * (t.nx + 1.), cy = .5 * (t.ny + 1.), cz = .5 * (t.nz + 1.);
        int expected = 0;
        long long q = 0;
        for (int i = 1; i <= t.nx; ++i)
            for (int j = 1; j <= t.ny; ++j)
                for (int k = 1; k <= (dim == 3 ? t.nz : 1); ++k, ++q) {
                    const double d2 = dim == 3 ? (i - cx) * (i - cx) + (j - cy) * (j - cy) + (k - cz) * (k - cz)
                                               : (i - cx) * (i - cx) + (j - cy) * (j - cy);
                    const bool inside = d2 <= t.radius_grid * t.radius_grid;
                    require(p[q] == double(inside), "center seed has exact voxel geometry");
                    expected += inside;
                }
        nicr_budget b;
        m.budget(&b);
        require(m.center_seed_cells == expected && b.nuclei == 1, "one center seed event");
        require(near(total(m, NICR_FIELD_O) - ld(b.initialO), ld(b.nucO)), "seed insertion budgets");
        int k = 0;
        m.nucleate(&k);
        require(k == 0, "center never triggers Ksp reseeding");
    }
    nicr_config t = c;
    t.grains = 0; t.radius_grid = 5.5;
    if (dim == 3) { t.nx = 31; t.ny = 25; t.nz = 23; }
    Model sphere(t);
    int cells = 0;
    sphere.stamp(dim == 3 ? 16 : 15, dim == 3 ? 13 : 12, dim == 3 ? 12 : 0, &cells);
    require(cells == (dim == 3 ? 739 : 97), dim == 3 ? "radius 5.5 sphere contains 739 voxels" : "R=5.5 disk has 97 sites, not R=5 disk");
    t = c;
    t.grains = 0; t.radius_grid = 2.5;
    Model wrap(t);
    wrap.stamp(12, 1, 1, &cells);
    const auto p = get(wrap, NICR_FIELD_PHI);
    if (dim == 3) {
        auto at = [&](int i, int j, int k) { return p[((size_t)(i - 1) * t.ny + (j - 1)) * t.nz + (k - 1)]; };
        require(at(12, t.ny, t.nz) == 1. && at(12, 2, 2) == 1., "sphere wraps both periodic seams");
    } else {
        require(p[(size_t)11 * t.ny + (t.ny - 1)] == 1. && p[(size_t)11 * t.ny + 1] == 1., "disk wraps the periodic seam");
    }
    t.nucleation = NICR_NUC_KSP;
    Model ksp(t);
    std::vector<double> o((size_t)ksp.g.ncells, .001);
    ksp.set_field(NICR_FIELD_O, 0, o.data());
    int nuclei = 0;
    ksp.nucleate(&nuclei);
    require(nuclei > 0, "Ksp hard-seed scan operates");
    std::cout << "PASS: " << dim << "D odd/even centre seeds, exact radius, seam wrapping and Ksp insertion.\n";
}

void test_eta(int dim) {
    nicr_config c = base(dim);
    c.grain_evolution = 1;
    Model eta(c);
    std::vector<double> sum((size_t)eta.g.ncells, 0.);
    for (int g = 0; g < eta.neta; ++g) {
        const auto e = get(eta, NICR_FIELD_ETA, g);
        for (size_t q = 0; q < sum.size(); ++q) sum[q] += e[q];
    }
    for (double s : sum) require(near(s, 1., 1.e-14L, 1.e-14L), "eta initialization partitions unity");
    require(near(eta.ec.scale, 1.), "eta auto width preserves integrated GB convention");
    nicr_config t = c;
    t.eta_L = 0.;
    Model frozen(t);
    std::vector<std::vector<double>> old;
    for (int g = 0; g < frozen.neta; ++g) old.push_back(get(frozen, NICR_FIELD_ETA, g));
    step(frozen, 5);
    for (int g = 0; g < frozen.neta; ++g) require(old[g] == get(frozen, NICR_FIELD_ETA, g), "eta-L=0 freezes eta PDE");
    int cells = 0;
    frozen.stamp(12, 1, 1, &cells);
    for (int g = 0; g < frozen.neta; ++g) {
        const auto e = get(frozen, NICR_FIELD_ETA, g);
        require(e[dim == 3 ? (size_t)11 * t.ny * t.nz : (size_t)11 * t.ny] == 0., "hard seeds consume eta even with eta-L=0");
    }
    // closed grain-only run: the discrete grain energy does not increase (3S:1230-1232)
    nicr_config e = c;
    if (dim == 3) { e.nx = 9; e.ny = 7; e.nz = 5; } else { e.nx = 17; e.ny = 13; }
    e.dx = e.dy = e.dz = 1.; e.grain_diameter_grid = 6.; e.eta_W = 2.; e.eta_kappa = .3; e.eta_L = .1; e.dt = 1.e-3;
    Model en(e);
    std::vector<double> z((size_t)en.g.ncells, 0.), cr((size_t)en.g.ncells, nicr::Phys::bulkCr);
    en.set_field(NICR_FIELD_O, 0, z.data());
    en.set_field(NICR_FIELD_CR, 0, cr.data());
    en.set_field(NICR_FIELD_PHI, 0, z.data());
    nicr_grain_stats gs;
    en.grain_stats(&gs, nullptr, nullptr);
    long double previous = ld(gs.energy);
    for (int n = 0; n < 30; ++n) {
        step(en);
        en.grain_stats(&gs, nullptr, nullptr);
        require(ld(gs.energy) <= previous + 1.e-12L, "closed grain-only energy is nonincreasing");
        previous = ld(gs.energy);
    }
    std::cout << "PASS: " << dim << "D eta initialization, frozen eta, seed consumption and energy descent.\n";
}

}  // namespace

namespace nicr {
int run_self_test(int dim) {
    try {
        std::cout << "GPU SELF-TEST: checks of the reference's built-in suite run on the CUDA model.\n";
        test_geometry(dim);
        test_transport(dim);
        test_seeds(dim);
        test_eta(dim);
        std::cout << "PASS: all " << dim << "D self-tests.\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << "\n";
        return 1;
    }
}
}  // namespace nicr
