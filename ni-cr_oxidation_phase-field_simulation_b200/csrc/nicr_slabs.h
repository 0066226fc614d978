// The slab form of one 3D domain (nicr_slabs.cpp): the group of X slabs, each
// a Model holding its planes plus neighbour halo planes, advanced together.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_model.h"

namespace nicr {

// Slab `index` of a domain split along X into n near-equal slabs (the first
// nx mod n slabs one plane longer) and the halo width: 2, or ceil(radius +
// gap) with Ksp nucleation (the reach of the pre-scan test).
SlabSpec slab_partition(const nicr_config& c, int n, int index);

class SlabGroup {
public:
    SlabGroup(const nicr_config& cfg, int n, const int* devices);
    ~SlabGroup();
    SlabGroup(const SlabGroup&) = delete;
    SlabGroup& operator=(const SlabGroup&) = delete;

    nicr_config c;
    int halo = 2;
    std::vector<std::unique_ptr<Model>> m;
    std::vector<int> x0, x1, dev;
    std::string err;

    int advance(int nsteps, bool schedule, int* completed);
    int nucleate(int* nuclei);
    void get_field(int field, int index, double* host);
    void set_field(int field, int index, const double* host);
    void reset_inventory();
    void budget(nicr_budget* b);
    void diagnostics(nicr_diagnostics* d);
    // grain_log values over all slabs (Model::grain_stats combined)
    void grain_stats(nicr_grain_stats* s, long long* cells, double* amount);
    // the seven 3D VTI arrays of the whole domain in file order (X fastest)
    // and type, gathered from the slabs' own planes; returns the out-of-range
    // bits of launch_vti_arrays
    unsigned vti_arrays(std::vector<unsigned char>& out, bool f64);
    size_t device_bytes() const;
    long long launches() const;

private:
    std::vector<cudaEvent_t> ev_done, ev_push;
    bool pushed = false;
    SlabPeers peers{};
    std::vector<KspNucleus*> d_pre, d_out;
    int cap = 1 << 16;                 // nuclei per slab and scan
    long long copies = 0;              // halo copy launches

    void on(int s) const { check_cuda(cudaSetDevice(dev[(size_t)s]), "cudaSetDevice"); }
    void one_step();
    void push(int s, bool step_fields, int p_width);
    void sync_all();
    bool any_failed();
    int scan();
};

}  // namespace nicr

// The group behind a C-ABI slab handle, and its last-error setter (for the
// entry points defined with the output code).
nicr::SlabGroup* nicr_slabs_group(nicr_slabs* h);
void nicr_slabs_set_error(nicr_slabs* h, const std::string& e);
