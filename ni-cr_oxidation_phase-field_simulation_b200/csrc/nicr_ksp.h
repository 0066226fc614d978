// Ksp nucleation: device parameter block, work buffers and launchers.
#pragma once
#include "nicr_kernels.h"

namespace nicr {

struct KspDev {
    Grid g;
    int nx, ny, nz;                 // reference extents (2D: ny = columns, nz = 1)
    double radius, gap, ksp;
    int neta;
    const unsigned char* hyp2d;     // 2D: hypot(|di|,|dj|) < r+gap, C-library hypot on the host
    int hyp_stride;
    const int* shadow;              // offsets within r+gap of a full ball (3 ints each)
    int n_shadow;
    const int* ball;                // ball offsets (3 ints each)
    int n_ball;
    int full_ball;                  // cells of an unclipped, unwrapped ball
    int box_half;                   // ceil(r) + ceil(r+gap)
    // X slab of a larger domain: stored plane 0 is domain plane x_off
    // (0-based); candidates and budget terms come from the own planes
    // [x_lo, x_hi) only. A whole domain: 0, 0, g.nx.
    int x_off, x_lo, x_hi;
};
// A nucleus of a scan in domain coordinates (1-based), full = its stamp set
// every cell of the ball (the exclusion marks are then the precomputed shadow).
struct KspNucleus {
    int x, y, z, full;
};
struct KspWork {
    unsigned char* flag;            // per cell: pre-scan candidate
    unsigned char* blocked;         // per cell: within r+gap of a cell stamped in this scan
    int* counts;                    // per compaction block
    long long* list;                // candidate cells in reference order
    int* total;
};
struct KspResult {
    int nuclei, last_cells, candidates, partial_stamps;
    int listed;                     // accepted nuclei of the scan (may exceed the list capacity)
    int pad;
};

int ksp_compact_blocks(long long ncells);
void launch_ksp_scan(const KspDev& K, double* o, double* cr, double* p, double* eta, KspWork& W, DevBudget* budget,
                     KspResult* res, Status* st, cudaStream_t stream);
void launch_ksp_stamp(const KspDev& K, int x, int y, int z, double* o, double* cr, double* p, double* eta,
                      KspWork& W, DevBudget* budget, KspResult* res, Status* st, cudaStream_t stream);
// Slab form of a scan (domain order = slab order along X):
//   launch_ksp_candidates   pre-scan test and ordered compaction of the own cells
//   launch_ksp_resolve_slab the ordered resolve: first the nuclei that slabs
//                           earlier in X accepted in this scan (pre, npre:
//                           their stamps on this slab's cells and their
//                           exclusion marks), then the own candidates; the
//                           accepted ones are listed in out (capacity cap,
//                           count in res->listed)
//   launch_ksp_apply        stamps of the nuclei that later slabs accepted
//                           (on this slab's cells, no marks)
void launch_ksp_candidates(const KspDev& K, const double* o, const double* cr, const double* p, KspWork& W,
                           Status* st, cudaStream_t stream);
void launch_ksp_resolve_slab(const KspDev& K, const KspNucleus* pre, int npre, KspNucleus* out, int cap, double* o,
                             double* cr, double* p, double* eta, KspWork& W, DevBudget* budget, KspResult* res,
                             Status* st, cudaStream_t stream);
void launch_ksp_apply(const KspDev& K, const KspNucleus* list, int n, double* o, double* cr, double* p, double* eta,
                      KspWork& W, DevBudget* budget, KspResult* res, Status* st, cudaStream_t stream);

}  // namespace nicr
