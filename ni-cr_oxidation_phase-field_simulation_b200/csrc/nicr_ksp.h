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
};

int ksp_compact_blocks(long long ncells);
void launch_ksp_scan(const KspDev& K, double* o, double* cr, double* p, double* eta, KspWork& W, DevBudget* budget,
                     KspResult* res, Status* st, cudaStream_t stream);
void launch_ksp_stamp(const KspDev& K, int x, int y, int z, double* o, double* cr, double* p, double* eta,
                      KspWork& W, DevBudget* budget, KspResult* res, Status* st, cudaStream_t stream);

}  // namespace nicr
