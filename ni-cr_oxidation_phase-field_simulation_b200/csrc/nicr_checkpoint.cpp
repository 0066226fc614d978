// Binary checkpoint / restart of one domain. The reference has none: its
// regression driver's snapshot_state (mpi3d-slab/tests/regression_driver.cpp:17-32)
// dumps the refreshed interior fields o, cr, p, muO, muCr, mo, mc, gb, eta_s2
// and every eta in (i, j, k) order, which is enough to compare states but not
// to resume a run. A checkpoint here is a header (magic, version, the
// configuration the state belongs to, step counter, nucleation clock, the
// budget and the Voronoi seeds), that same field section in that same order
// and layout, then the fields a resume needs beyond it (the grain map when it
// is kept, the 2D initial GB mask) and a 64-bit FNV-1a checksum of all bytes
// before it. Loading it into a handle made from the same configuration
// restores a state from which stepping continues bit for bit as if the run
// had not been interrupted.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "nicr_model.h"

namespace nicr {
namespace {

constexpr char kMagic[8] = {'N', 'I', 'C', 'R', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 1;

struct Header {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    nicr_config cfg;
    long long steps_done;
    double next_nucleation;
    int dim, neta, has_eta, grain_retained, center_seed_cells, n_seeds;
    nicr_budget budget;
};

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
    }
};

struct Out {
    std::ofstream f;
    Fnv sum;
    explicit Out(const std::string& path) : f(path, std::ios::binary | std::ios::trunc) {}
    void put(const void* p, size_t n) {
        f.write(static_cast<const char*>(p), (std::streamsize)n);
        sum.add(p, n);
    }
};

struct In {
    std::ifstream f;
    Fnv sum;
    explicit In(const std::string& path) : f(path, std::ios::binary) {}
    bool get(void* p, size_t n) {
        f.read(static_cast<char*>(p), (std::streamsize)n);
        if (!f) return false;
        sum.add(p, n);
        return true;
    }
};

// Configuration fields that decide the evolution of a state; everything else
// (run length, output cadence and format, device, arithmetic form) may differ
// between the run that wrote a checkpoint and the one that resumes it.
std::string config_mismatch(const nicr_config& a, const nicr_config& b) {
#define NICR_SAME(f) if (std::memcmp(&a.f, &b.f, sizeof a.f) != 0) return #f;
    NICR_SAME(dim) NICR_SAME(nx) NICR_SAME(ny)
    if (a.dim == 3) { NICR_SAME(nz) }
    NICR_SAME(left_edge_sites) NICR_SAME(max_eta_fields) NICR_SAME(random_seed)
    NICR_SAME(dx) NICR_SAME(dy) NICR_SAME(dz) NICR_SAME(dt) NICR_SAME(grain_diameter_grid) NICR_SAME(gb_fwhm_grid)
    NICR_SAME(gb_factor_o) NICR_SAME(gb_factor_cr) NICR_SAME(radius_grid) NICR_SAME(exclusion_gap_grid)
    NICR_SAME(nucleation_period) NICR_SAME(mu_res) NICR_SAME(surface_c_ref) NICR_SAME(bc) NICR_SAME(ck)
    NICR_SAME(bounds) NICR_SAME(nucleation) NICR_SAME(grains) NICR_SAME(oxygen_diffusion) NICR_SAME(grain_evolution)
    NICR_SAME(frozen_eta_cache) NICR_SAME(eta_W) NICR_SAME(eta_kappa) NICR_SAME(eta_L) NICR_SAME(eta_oxide_penalty)
    NICR_SAME(ksp) NICR_SAME(bulk_cr) NICR_SAME(layer_o) NICR_SAME(eta_colours)
#undef NICR_SAME
    return "";
}

}  // namespace

void Model::save_state(const std::string& path) {
    refresh();   // mu and M of the current state, as the reference's snapshot does
    Header h{};
    std::memcpy(h.magic, kMagic, sizeof kMagic);
    h.version = kVersion;
    h.header_bytes = (uint32_t)sizeof(Header);
    h.cfg = c;
    h.steps_done = steps_done;
    h.next_nucleation = next_nucleation;
    h.dim = dim;
    h.neta = neta;
    h.has_eta = has_eta ? 1 : 0;
    h.grain_retained = grain_retained ? 1 : 0;
    h.center_seed_cells = center_seed_cells;
    h.n_seeds = (int)volumes.size();
    budget(&h.budget);
    Out o(path);
    if (!o.f) throw Error(NICR_ERR_IO, "Cannot open checkpoint for writing: " + path);
    o.put(&h, sizeof h);
    o.put(seeds.data(), seeds.size() * sizeof(double));
    o.put(volumes.data(), volumes.size() * sizeof(long long));
    std::vector<double> host((size_t)g.ncells);
    auto field = [&](const double* d) {
        copy_out(d, host.data());
        o.put(host.data(), host.size() * sizeof(double));
    };
    // the reference's snapshot_state section: o cr p muO muCr mo mc gb [eta_s2] eta...
    for (const double* d : {o_[cur], cr_[cur], p_[cur], muO, muCr, mo, mc, gb_[gcur]}) field(d);
    if (has_eta) field(s2_[gcur]);
    for (int q = 0; q < neta; ++q) field(eta_[ecur] + (size_t)q * g.nstore);
    // beyond it: what a resume needs
    if (grain_retained) field(grain);
    if (dim == 2) field(gb_initial);
    const uint64_t sum = o.sum.h;
    o.f.write(reinterpret_cast<const char*>(&sum), sizeof sum);
    o.f.flush();
    if (!o.f) throw Error(NICR_ERR_IO, "Checkpoint write failed: " + path);
}

void Model::load_state(const std::string& path) {
    In in(path);
    if (!in.f) throw Error(NICR_ERR_IO, "Cannot open checkpoint: " + path);
    Header h{};
    if (!in.get(&h, sizeof h) || std::memcmp(h.magic, kMagic, sizeof kMagic) != 0)
        throw Error(NICR_ERR_INVALID_ARG, "Not a checkpoint of this library: " + path);
    if (h.version != kVersion || h.header_bytes != sizeof(Header))
        throw Error(NICR_ERR_INVALID_ARG, "Unsupported checkpoint version in " + path);
    const std::string bad = config_mismatch(h.cfg, c);
    if (!bad.empty())
        throw Error(NICR_ERR_INVALID_ARG, "Checkpoint " + path + " belongs to another configuration (" + bad + " differs)");
    if (h.dim != dim || h.neta != neta || (h.has_eta != 0) != has_eta || (h.grain_retained != 0) != grain_retained ||
        h.n_seeds != (int)volumes.size())
        throw Error(NICR_ERR_INVALID_ARG, "Checkpoint " + path + " does not match this domain's layout");
    std::vector<double> sd(seeds.size());
    std::vector<long long> vol(volumes.size());
    if (!in.get(sd.data(), sd.size() * sizeof(double)) || !in.get(vol.data(), vol.size() * sizeof(long long)))
        throw Error(NICR_ERR_INVALID_ARG, "Truncated checkpoint: " + path);
    const size_t nf = 8 + (has_eta ? 1 : 0) + (size_t)neta + (grain_retained ? 1 : 0) + (dim == 2 ? 1 : 0);
    std::vector<double> all(nf * (size_t)g.ncells);
    if (!in.get(all.data(), all.size() * sizeof(double))) throw Error(NICR_ERR_INVALID_ARG, "Truncated checkpoint: " + path);
    uint64_t stored = 0;
    const uint64_t computed = in.sum.h;
    in.f.read(reinterpret_cast<char*>(&stored), sizeof stored);
    if (!in.f || stored != computed) throw Error(NICR_ERR_INVALID_ARG, "Checkpoint checksum mismatch: " + path);

    // everything verified: install the state
    auto at = [&](size_t k) { return all.data() + k * (size_t)g.ncells; };
    copy_in(o_[cur], at(0));
    copy_in(cr_[cur], at(1));
    copy_in(p_[cur], at(2));
    copy_in(gb_[gcur], at(7));           // fields 3..6 (mu, M) are derived: refresh() recomputes them
    size_t k = 8;
    if (has_eta) copy_in(s2_[gcur], at(k++));
    for (int q = 0; q < neta; ++q) copy_in(eta_[ecur] + (size_t)q * g.nstore, at(k++));
    if (grain_retained) copy_in(grain, at(k++));
    if (dim == 2) copy_in(gb_initial, at(k++));
    seeds = sd;
    volumes = vol;
    center_seed_cells = h.center_seed_cells;
    DevBudget b{};
    const nicr_budget& nb = h.budget;
    const double* src[8] = {nb.nucO, nb.nucCr, nb.ckO, nb.ckCr, nb.clipO, nb.clipCr, nb.bcO, nb.bcCr};
    for (int q = 0; q < 8; ++q) { b.v[q][0] = src[q][0]; b.v[q][1] = src[q][1]; }
    b.nuclei = nb.nuclei;
    b.clipped = nb.clipped;
    b.initialO[0] = nb.initialO[0]; b.initialO[1] = nb.initialO[1];
    b.initialCr[0] = nb.initialCr[0]; b.initialCr[1] = nb.initialCr[1];
    check_cuda(cudaMemcpyAsync(bud, &b, sizeof b, cudaMemcpyHostToDevice, stream), "H2D");
    steps_done = h.steps_done;
    next_nucleation = h.next_nucleation;
    eta_dirty = false;   // gb and eta_s2 are the saved (refreshed) mask of the saved eta
    sync();
    refresh();
}

}  // namespace nicr
