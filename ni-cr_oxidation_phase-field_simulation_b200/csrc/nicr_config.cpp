// Configuration defaults and the command-line parser of the solver programs.
// Same flags, defaults, validation order and error messages as the
// reference's parse() (2D:712-790, 3S:980-1082); the help text is this
// program's own.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/nicr.h"
#include "nicr_physics.h"

namespace {

constexpr const char* VERSION2 = "mpi-eta-v1";                     // 2D:38
constexpr const char* VERSION3 = "mpi-eta-3d-xslab-optimized-v1";  // 3S:41

struct Early {
    std::string text;
};

bool on_off(const std::string& v, const std::string& opt) {
    if (v == "on") return true;
    if (v == "off") return false;
    throw std::runtime_error(opt + " expects on or off (received: " + v + ")");
}

std::string help_text(int dim) {
    std::string s =
        "Initialization only by default (no steps). Options:\n"
        "--steps N --dt s --nx N --ny N" + std::string(dim == 3 ? " --nz N" : "") +
        " --dx m (all spacings) --output-every N\n"
        "--grains on|off            Voronoi metal grains with GB-enhanced transport (default on)\n"
        "--grain-evolution on|off   evolving eta order parameters (default off)\n"
        "--eta-W v --eta-kappa v (0: auto) --eta-L v --eta-oxide-penalty v (-1: eta-W)\n"
        "--eta-output all|summary --max-eta-fields N (default 512)\n";
    if (dim == 3)
        s += "--output-format vti|vtk --output-precision float32|float64 --compression-level 0..9\n"
             "--frozen-eta-cache on|off\n";
    s += "--oxygen-diffusion on|off  O transport and O boundary supply (default on)\n"
         "--left-edge-sites N" + std::string(dim == 3 ? " (alias --left-face-sites)" : "") +
         "  anchor N Voronoi sites on the inlet face\n"
         "--grain-diameter-grid N --gb-width-grid N --gb-factor-o N --gb-factor-cr N [--gb-factor N] --seed N\n"
         "--nucleation ksp|center|off --radius-grid R --nucleation-period s\n"
         "--bc concentration|mu|closed --mu-res v --surface-c-ref v\n"
         "--ck legacy|off --bounds stop|legacy --out directory --self-test --version\n"
         "Extensions (defaults reproduce the fixed reference constants): --ksp v --bulk-cr v --layer-o v\n"
         "--precision fp64|fp64-fast (fp64: bit-identical to the reference; fp64-fast: reciprocal divisions)\n"
         "--checkpoint-every N (write <out>/checkpoint.bin every N steps) --restart FILE (continue from a checkpoint)\n";
    if (dim == 3)
        s += "--eta-colours K (evolving grains: colour the Voronoi grains into K eta fields with tanh boundaries)\n"
             "--slabs N [--slab-devices a,b,...] (the domain split along X over N slabs/GPUs; VTI output only)\n";
    return s;
}

double eta_K_of(const nicr_config& c) {
    return nicr::eta_coef(c.gb_fwhm_grid, c.dx, c.eta_W, c.eta_kappa, c.eta_oxide_penalty).K;
}
double eta_scale_of(const nicr_config& c) {
    return nicr::eta_coef(c.gb_fwhm_grid, c.dx, c.eta_W, c.eta_kappa, c.eta_oxide_penalty).scale;
}

void parse_into(nicr_config& c, int dim, int argc, const char* const* argv, std::string& out, bool& self_test) {
    std::string eta_output = "all", fmt = "vti", prec = "float32";
    for (int q = 0; q < argc; ++q) {
        const std::string a = argv[q];
        if (a == "--self-test") { self_test = true; continue; }
        if (a == "--version") throw Early{std::string(dim == 3 ? VERSION3 : VERSION2) + "\n"};
        if (a == "--help") throw Early{help_text(dim)};
        if (q + 1 >= argc) throw std::runtime_error("Missing value for " + a);
        const std::string v = argv[++q];
        if (a == "--steps") c.steps = std::stoi(v);
        else if (a == "--dt") c.dt = std::stod(v);
        else if (a == "--nx") c.nx = std::stoi(v);
        else if (a == "--ny") c.ny = std::stoi(v);
        else if (dim == 3 && a == "--nz") c.nz = std::stoi(v);
        else if (a == "--dx") { c.dx = c.dy = std::stod(v); if (dim == 3) c.dz = c.dx; }
        else if (a == "--output-every") c.output_every = std::stoi(v);
        else if (a == "--grains") c.grains = on_off(v, a);
        else if (a == "--grain-evolution") c.grain_evolution = on_off(v, a);
        else if (a == "--eta-W") c.eta_W = std::stod(v);
        else if (a == "--eta-kappa") c.eta_kappa = std::stod(v);
        else if (a == "--eta-L") c.eta_L = std::stod(v);
        else if (a == "--eta-oxide-penalty") c.eta_oxide_penalty = std::stod(v);
        else if (a == "--eta-output") eta_output = v;
        else if (a == "--max-eta-fields") c.max_eta_fields = std::stoi(v);
        else if (dim == 3 && a == "--output-format") fmt = v;
        else if (dim == 3 && a == "--output-precision") prec = v;
        else if (dim == 3 && a == "--compression-level") {
            std::size_t used = 0;
            c.compression_level = std::stoi(v, &used);
            if (used != v.size()) throw std::runtime_error("--compression-level expects an integer 0..9.");
        } else if (dim == 3 && a == "--frozen-eta-cache") c.frozen_eta_cache = on_off(v, a);
        else if (a == "--oxygen-diffusion") c.oxygen_diffusion = on_off(v, a);
        else if (a == "--left-edge-sites" || (dim == 3 && a == "--left-face-sites")) {
            std::size_t used = 0;
            c.left_edge_sites = std::stoi(v, &used);
            if (used != v.size() || c.left_edge_sites < 0)
                throw std::runtime_error("--left-edge-sites expects a nonnegative integer.");
        } else if (a == "--grain-diameter-grid") c.grain_diameter_grid = std::stod(v);
        else if (a == "--gb-width-grid") c.gb_fwhm_grid = std::stod(v);
        else if (a == "--gb-factor-o") c.gb_factor_o = std::stod(v);
        else if (a == "--gb-factor-cr") c.gb_factor_cr = std::stod(v);
        else if (a == "--gb-factor") { c.gb_factor_o = std::stod(v); c.gb_factor_cr = c.gb_factor_o; }
        else if (a == "--nucleation") {
            if (v == "ksp") c.nucleation = NICR_NUC_KSP;
            else if (v == "center") c.nucleation = NICR_NUC_CENTER;
            else if (v == "off") c.nucleation = NICR_NUC_OFF;
            else c.nucleation = -1;
        } else if (a == "--radius-grid") c.radius_grid = std::stod(v);
        else if (a == "--nucleation-period") c.nucleation_period = std::stod(v);
        else if (a == "--seed") c.random_seed = std::stoull(v);
        else if (a == "--bc") c.bc = v == "concentration" ? NICR_BC_CONCENTRATION : v == "mu" ? NICR_BC_MU : v == "closed" ? NICR_BC_CLOSED : -1;
        else if (a == "--ck") c.ck = v == "legacy" ? NICR_CK_LEGACY : v == "off" ? NICR_CK_OFF : -1;
        else if (a == "--bounds") c.bounds = v == "stop" ? NICR_BOUNDS_STOP : v == "legacy" ? NICR_BOUNDS_LEGACY : -1;
        else if (a == "--out") out = v;
        else if (a == "--mu-res") c.mu_res = std::stod(v);
        else if (a == "--surface-c-ref") c.surface_c_ref = std::stod(v);
        else if (a == "--ksp") c.ksp = std::stod(v);
        else if (a == "--bulk-cr") c.bulk_cr = std::stod(v);
        else if (a == "--layer-o") c.layer_o = std::stod(v);
        else if (a == "--checkpoint-every") {
            size_t used = 0;
            const long long n = std::stoll(v, &used);
            if (used != v.size() || n < 0 || n > INT_MAX)
                throw std::runtime_error("--checkpoint-every expects a nonnegative integer.");
            c.checkpoint_every = (int)n;
        }
        else if (a == "--eta-colours" && dim == 3) {
            size_t used = 0;
            const long long n = std::stoll(v, &used);
            if (used != v.size() || n < 0 || n > 4096) throw std::runtime_error("--eta-colours expects an integer in [0, 4096].");
            c.eta_colours = (int)n;
        }
        else if (a == "--precision") {
            if (v == "fp64") c.precision = NICR_FP64;
            else if (v == "fp64-fast") c.precision = NICR_FP64_FAST;
            else throw std::runtime_error("--precision expects fp64 or fp64-fast.");
        }
        else throw std::runtime_error("Unknown argument: " + a);
    }
    // validation, in the reference's order (3S:1055-1081, 2D:770-789)
    const double finite_list[] = {c.dx, c.dy, dim == 3 ? c.dz : c.dy, c.dt, c.grain_diameter_grid, c.gb_fwhm_grid,
                                  c.gb_factor_o, c.gb_factor_cr, c.radius_grid, c.nucleation_period, c.mu_res,
                                  c.surface_c_ref, c.ksp, c.bulk_cr, c.layer_o};
    for (double x : finite_list)
        if (!std::isfinite(x)) throw std::runtime_error("All numerical parameters must be finite.");
    const bool bad_dims = dim == 3 ? (c.nx < 3 || c.ny < 3 || c.nz < 3 || c.nx > INT_MAX - 2 || c.ny > INT_MAX - 2 || c.nz > INT_MAX - 2)
                                   : (c.nx < 3 || c.ny < 3 || c.nx > INT_MAX - 2 || c.ny > INT_MAX - 2);
    if (bad_dims || c.steps < 0 || c.output_every < 1 || c.dt <= 0 || c.dx <= 0 || c.dy <= 0 || (dim == 3 && c.dz <= 0) ||
        c.grain_diameter_grid <= 0 || c.gb_fwhm_grid <= 0 || c.gb_factor_o < 1 || c.gb_factor_cr < 1 || c.radius_grid <= 0 ||
        (c.nucleation == NICR_NUC_KSP && c.nucleation_period < c.dt) || c.nucleation_period <= 0. || c.surface_c_ref <= 0)
        throw std::runtime_error("Invalid parameter bounds (Ksp nucleation period must be >= dt).");
    for (double v : {c.eta_W, c.eta_kappa, c.eta_L, c.eta_oxide_penalty})
        if (!std::isfinite(v)) throw std::runtime_error("Eta parameters must be finite.");
    if (c.eta_W <= 0. || c.eta_kappa < 0. || c.eta_L < 0. || (c.eta_oxide_penalty < 0. && c.eta_oxide_penalty != -1.) ||
        c.max_eta_fields < 1)
        throw std::runtime_error("Invalid eta parameter bounds.");
    if (dim == 3) {
        if (fmt != "vti" && fmt != "vtk") throw std::runtime_error("--output-format expects vti or vtk.");
        if (prec != "float32" && prec != "float64") throw std::runtime_error("--output-precision expects float32 or float64.");
        if (c.compression_level < 0 || c.compression_level > 9) throw std::runtime_error("--compression-level must lie in [0,9].");
        if (!std::isfinite(c.exclusion_gap_grid) || c.exclusion_gap_grid < 0. || !std::isfinite(c.radius_grid + c.exclusion_gap_grid))
            throw std::runtime_error("Nucleation exclusion length must be finite and nonnegative.");
    }
    if (eta_output != "all" && eta_output != "summary") throw std::runtime_error("--eta-output expects all or summary.");
    if (c.grain_evolution && c.grains && (!std::isfinite(eta_K_of(c)) || !std::isfinite(eta_scale_of(c)) || eta_K_of(c) <= 0.))
        throw std::runtime_error("Derived eta coefficients are invalid.");
    if (c.nucleation < 0) throw std::runtime_error("--nucleation expects ksp, center, or off.");
    if (dim == 3) {
        if (c.nucleation == NICR_NUC_CENTER && c.radius_grid >= 0.5 * (double(std::min({c.nx, c.ny, c.nz})) - 1.))
            throw std::runtime_error("Center seed is too large: --radius-grid must be less than (min(nx,ny,nz)-1)/2.");
        if (c.nucleation == NICR_NUC_KSP && c.radius_grid >= 0.5 * std::min(c.ny, c.nz))
            throw std::runtime_error("Ksp sphere radius must be less than min(ny,nz)/2 to avoid periodic self-overlap.");
    } else if (c.nucleation == NICR_NUC_CENTER && c.radius_grid >= 0.5 * (double(std::min(c.nx, c.ny)) - 1.)) {
        throw std::runtime_error("Center seed is too large: --radius-grid must be less than (min(nx,ny)-1)/2.");
    }
    if (c.bc < 0) throw std::runtime_error("Invalid bc.");
    if (c.ck < 0) throw std::runtime_error("Invalid Ck mode.");
    if (c.bounds < 0) throw std::runtime_error("Invalid bounds mode.");
    c.eta_output_all = eta_output == "all";
    c.output_vti = fmt == "vti";
    c.output_float64 = prec == "float64";
}

void copy_str(char* dst, size_t len, const std::string& s) {
    if (!dst || len == 0) return;
    std::strncpy(dst, s.c_str(), len - 1);
    dst[len - 1] = 0;
}

}  // namespace

extern "C" void nicr_config_default(nicr_config* c, int dim) {
    std::memset(c, 0, sizeof *c);
    c->dim = dim;
    c->nx = 151; c->ny = 101; c->nz = dim == 3 ? 101 : 1;
    c->steps = 0; c->output_every = 5000;
    c->left_edge_sites = 0;
    c->max_eta_fields = 512;
    c->random_seed = 20260909ULL;
    c->dx = c->dy = c->dz = 1.e-8;
    c->dt = 2e-10;
    c->grain_diameter_grid = 50.; c->gb_fwhm_grid = 4.;
    c->gb_factor_o = 28.2; c->gb_factor_cr = 563.;
    c->radius_grid = 5.5; c->exclusion_gap_grid = 6.; c->nucleation_period = 1.e-7;
    c->mu_res = 364688.; c->surface_c_ref = 0.0023;
    c->bc = NICR_BC_CONCENTRATION; c->ck = NICR_CK_LEGACY; c->bounds = NICR_BOUNDS_STOP; c->nucleation = NICR_NUC_KSP;
    c->grains = 1; c->oxygen_diffusion = 1; c->grain_evolution = 0; c->frozen_eta_cache = 1;
    c->eta_W = 1.e4; c->eta_kappa = 0.; c->eta_L = 0.2; c->eta_oxide_penalty = -1.;
    c->eta_output_all = 1;
    c->output_vti = 1; c->output_float64 = 0; c->compression_level = 1;
    c->ksp = nicr::Phys::ksp; c->bulk_cr = nicr::Phys::bulkCr; c->layer_o = nicr::Phys::layerO;
    c->precision = NICR_FP64;
    c->device = 0;
}

extern "C" int nicr_config_parse(nicr_config* cfg, int dim, int argc, const char* const* argv, char* out_dir,
                                 size_t out_dir_len, int* self_test, char* err, size_t err_len) {
    if (!cfg || (dim != 2 && dim != 3)) return NICR_ERR_INVALID_ARG;
    nicr_config c;
    nicr_config_default(&c, dim);
    std::string out = dim == 3 ? "nicr3d_grains_output" : "nicr_grains_output";
    bool st = false;
    try {
        parse_into(c, dim, argc, argv, out, st);
    } catch (const Early& e) {
        copy_str(err, err_len, e.text);
        return 100;
    } catch (const std::exception& e) {
        copy_str(err, err_len, e.what());
        return NICR_ERR_INVALID_ARG;
    }
    *cfg = c;
    copy_str(out_dir, out_dir_len, out);
    if (self_test) *self_test = st ? 1 : 0;
    return NICR_OK;
}
