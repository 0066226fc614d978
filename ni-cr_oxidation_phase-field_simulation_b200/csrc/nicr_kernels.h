// Launch interface between the host model (g++) and the CUDA kernels (nvcc).
// Plain C++: parameter blocks passed by value to the kernels, and launchers.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

#include "nicr_physics.h"

namespace nicr {

// Device layout of one field. X (planes) is slowest like the reference
// (3S:165-167); inside a plane, rows (3D: Y) then columns (3D: Z, 2D: Y), the
// column pitch padded to a multiple of 8 doubles so that every row starts on a
// 64-byte boundary. No ghost cells are stored: the kernels apply Neumann X and
// periodic row/column boundaries while staging tiles.
struct Grid {
    int dim;          // 2 or 3
    int nx;           // planes (reference X)
    int na;           // rows: 3D ny, 2D 1
    int nb;           // columns: 3D nz, 2D ny
    int pb;           // padded column pitch (elements)
    long long plane;  // na * pb
    long long ncells; // nx * na * nb
    long long nstore; // nx * plane
};

// Device status word of one domain: sticky failure flag, first failing trial
// (minimum key in reference loop order), step counters.
struct Status {
    unsigned long long err_key;   // ERR_NONE when no trial failed this step
    int failed;                   // a step of this batch was rejected
    int timeout;                  // a kernel's bounded wait for its own copies ran out
    long long failed_step;        // index (steps_done) of the rejected step
    long long steps_done;         // accepted steps since creation
    // Slab form: first failing trial of the step that reads buffer parity q,
    // in slot q (the slabs of a domain agree on a step's outcome by reading
    // every slab's slot of that step; see launch_step_finalize_slab).
    unsigned long long slot_err[2];
};
constexpr unsigned long long ERR_NONE = ~0ull;
constexpr unsigned long long ERR_ETA_BASE = 1ull << 62;

// Budget in double-double (Budget, 3S:217); order nucO nucCr ckO ckCr clipO clipCr bcO bcCr
struct DevBudget {
    double v[8][2];
    long long nuclei, clipped;
    double initialO[2], initialCr[2];
};

// Per-CTA partial sums of one step (ckO ckCr clipO clipCr bcO as hi/lo) + clipped count
struct StepPartial {
    double s[5][2];
    long long clipped;
    int redo;   // drop-in form: the CTA's chunk awaits the recomputation kernel
    int pad;
};

struct StepParams {
    Grid g;
    double dx, da, db, dt;       // spacing along X, rows, columns
    double dxdx, dada, dbdb;     // c.dx*c.dx etc. (lap denominators, 3S:193-195)
    DivC v_dxdx, v_dada, v_dbdb, v_dx, v_da, v_db, v_dt;  // exact divisions by the same constants
    double dtL;                  // dt * Physics::L
    double layer_o;
    double gbm1_o, gbm1_cr;      // gb_factor_o - 1, gb_factor_cr - 1
    double mu_res, surface_c_ref;
    double eta_W, eta_A, eta_K, dt_etaL, eta_scale;
    int bc, ck, bounds;
    int o_on;                    // oxygen_diffusion
    int grains;                  // GB mask active in mobility
    int phi_eta;                 // eta coupling in the phi force (has_eta)
    int inlet;                   // bc == concentration && oxygen_diffusion
    int xchunk;                  // planes per CTA along X
    int fast;                    // arithmetic form: 0 drop-in (bit-identical), 1 reciprocal divisions
    int minb;                    // 3D step kernel: CTAs/SM variant 2 or 3 (0: the default)
    // Planes updated: [x_lo, x_hi) of the g.nx stored planes. A whole domain
    // updates all of them; an X slab of a larger domain stores halo planes
    // below and above its own, which the kernels read but do not write.
    int x_lo, x_hi;
    // Failing-trial keys in whole-domain reference order: the cell index is
    // offset by cell_off and eta keys count key_ncells cells per field.
    long long cell_off, key_ncells;
    // Error word of this step: -1 st->err_key, 0/1 st->slot_err[err_slot] (slab form)
    int err_slot, pad_;
};
// The whole-domain values of the range fields (every plane, no offset).
inline void whole_domain_range(StepParams& sp) {
    sp.x_lo = 0;
    sp.x_hi = sp.g.nx;
    sp.cell_off = 0;
    sp.key_ncells = sp.g.ncells;
    sp.err_slot = -1;
}

// ---- step --------------------------------------------------------------------
// Main fused step: mu, M, six-face fluxes, phi, Ck, bounds -> trial buffers.
void launch_step_main(const StepParams& P, const double* o, const double* cr, const double* p,
                      const double* gb, const double* s2, double* on, double* crn, double* pn,
                      StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out);
int step_main_blocks(const StepParams& P);
// kernels launch_step_main launches: the drop-in form adds the recomputation
// kernel of CTAs whose numerators left the exact-division range
int step_main_kernels(const StepParams& P);
// Planes per CTA along X for grid g (step and eta kernels), and one chunk for
// the n domains of a batch. NICR_XCHUNK forces a chunk for tuning runs.
int choose_xchunk(const Grid& g);
// The same choice for the one-pass step (16 x 32 tiles, one CTA per SM).
int choose_xchunk_fused(const Grid& g);
int choose_xchunk_batch(const Grid* grids, int n);
// The chunks the choosers consider for a largest X extent nxmax: nxmax halved
// repeatedly and the powers of two below it, longest first.
std::vector<int> xchunk_candidates(int nxmax);
// Per-device kernel attributes of the step kernel P selects, set outside any
// stream capture (launch_step_main sets them on first use otherwise).
void step_kernels_prepare(const StepParams& P);
// The reciprocal form's launchers (nicr_step_fast.cu, compiled with FMA
// contraction); the generic launchers dispatch to them when P.fast is set.
void launch_step_main_fast(const StepParams& P, const double* o, const double* cr, const double* p, const double* gb,
                           const double* s2, double* on, double* crn, double* pn, StepPartial* partials, Status* st,
                           cudaStream_t stream, int* nblocks_out);
void launch_eta_update_fast(const StepParams& P, int neta, const double* eta, const double* s2, const double* p,
                            double* eta_next, double* gb_next, double* s2_next, Status* st, cudaStream_t stream);
void step_kernels_prepare_fast(const StepParams& P);
// Eta mask: S = sum eta^2, pairs, gb = scale*min(1,16*pairs) (3S:495-507)
void launch_eta_mask(const StepParams& P, int neta, const double* eta, double* gb, double* s2,
                     double* pairs, Status* st, cudaStream_t stream);
// Eta trial update (3S:514-526) + next-step mask from the trial values
void launch_eta_update(const StepParams& P, int neta, const double* eta, const double* s2,
                       const double* p, double* eta_next, double* gb_next, double* s2_next,
                       Status* st, cudaStream_t stream);
// Batched step of many domains in one launch per group of <= kBatchMax domains
// of one dimensionality and arithmetic form (consecutive entries). Each entry
// carries the domain's parameters and buffers; gx, gy, block0 are filled by the
// launcher, nblocks (the domain's partial-sum count) is written back.
struct BatchDomain {
    StepParams sp;
    const double *o, *cr, *p, *gb, *s2;
    double *on, *crn, *pn;
    StepPartial* partials;
    Status* st;
    int gx, gy, block0, nblocks;
};
constexpr int kBatchMax = 48;   // 48 entries: ~24 KB of kernel parameters (limit 32 KB)
struct StepBatch {
    int n, pad;
    BatchDomain d[kBatchMax];
};
// Compact form of a batch whose domains share every step parameter except
// the grid, the inlet value and the plane/key ranges that follow from the
// grid (a parameter sweep over sizes, O supply, Cr and Ksp, which the step
// kernel does not read): the shared parameters once, ~170 bytes per domain,
// so one launch serves up to kBatchSlimMax domains.
struct BatchSlim {
    Grid g;
    double layer_o;
    long long key_ncells;
    int x_hi, inlet, gx, gy, block0, pad;
    const double *o, *cr, *p, *gb, *s2;
    double *on, *crn, *pn;
    StepPartial* partials;
    Status* st;
};
constexpr int kBatchSlimMax = 160;   // 160 x 168 bytes + the shared parameters: < 27.5 KB of kernel parameters
struct StepBatchSlim {
    StepParams base;
    int n, pad;
    BatchSlim d[kBatchSlimMax];
};
// returns the number of launches: one for the whole batch in the compact
// form when it applies, else one per group of kBatchMax domains
int launch_step_batch(BatchDomain* doms, int n, cudaStream_t stream);
void launch_batch_slim_fast(const StepBatchSlim& B, int nblocks, int dim, cudaStream_t stream);
void launch_batch_group_fast(StepBatch& B, int nblocks, int dim, cudaStream_t stream);

// One launch for the step kernel and the eta update of one step (reciprocal
// form, 3D, 1..16 eta fields): the two are independent within a step, and
// their CTAs share the SMs (see k_step_eta). ticket: one word of device
// memory, zeroed by the launcher before each launch. Returns false (nothing
// launched) when the form does not apply; nblocks_out receives the step
// kernel's partial-sum count.
bool launch_step_eta_fast(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                          const double* gb, const double* s2, double* on, double* crn, double* pn,
                          StepPartial* partials, const double* eta, double* eta_next, double* gb_next,
                          double* s2_next, unsigned* ticket, Status* st, cudaStream_t stream, int* nblocks_out);
void step_eta_prepare_fast(const StepParams& P, int neta);

// One HBM pass per step (3D, evolving eta): the step kernel and the eta
// update fused into one X march with the eta planes staged by TMA and S / gb
// rebuilt on chip (k_step_fused, nicr_step_fused.cuh). It reads o, cr, p and
// the n eta fields and writes the trial o, cr, p and eta; gb and eta_s2 are
// neither read nor written. Applies to 1 <= n <= 8 fields, rows a multiple of
// 16 and columns a multiple of 32 (step_fused_applies); the launchers return
// false and launch nothing otherwise. The drop-in form is bit-identical to
// the two-kernel form.
bool step_fused_applies(const Grid& g, int neta);
bool launch_step_fused(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                       const double* eta, double* on, double* crn, double* pn, double* eta_next,
                       StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out);
bool launch_step_fused_fast(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                            const double* eta, double* on, double* crn, double* pn, double* eta_next,
                            StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out);
// kernel attributes of the fused step, set outside any stream capture
void step_fused_prepare(const StepParams& P, int neta);
void step_fused_prepare_fast(const StepParams& P, int neta);

struct FinalizeDomain {
    const StepPartial* partials;
    int nblocks, pad;
    DevBudget* budget;
    Status* st;
};
constexpr int kFinalizeMax = 512;
struct FinalizeBatch {
    int n, pad;
    FinalizeDomain d[kFinalizeMax];
};
void launch_finalize_batch(const FinalizeDomain* doms, int n, cudaStream_t stream);

// The seven arrays of a 3D VTI frame in file order (X fastest) and type, for
// the output path (nicr_vti.cu). range gets bit a set when array a holds a
// finite value outside the Float32 range.
struct VtiArgs {
    Grid g;
    int has_eta, neta;
    const double *p, *o, *cr, *muO, *muCr, *gb, *grain, *eta;
};
void launch_vti_arrays(const VtiArgs& a, void* out, bool f64, unsigned* range, cudaStream_t stream);

// Commit of one step: reduce partials, commit budget unless a trial failed
void launch_step_finalize(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st,
                          int accept_mode, cudaStream_t stream);
// Slab form of the commit: the step is rejected when any slab's error word
// of this step (peers[j]->slot_err[slot], read after every slab's step
// kernels completed) holds a failing trial; the minimum key is recorded in
// st->err_key. peers may live on other GPUs (peer access enabled).
constexpr int kMaxSlabs = 16;
struct SlabPeers {
    const Status* st[kMaxSlabs];
    int n, slot;
};
void launch_step_finalize_slab(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st,
                               const SlabPeers& peers, cudaStream_t stream);
// One process per slab: the slab's error word of the step (slot) as a signed
// agreement word (kAgreeNone when every trial passed, else the key), which
// the ranks reduce with a MIN collective; the commit then reads the result.
constexpr long long kAgreeNone = 0x7fffffffffffffffLL;
void launch_agree_word(const Status* st, int slot, long long* agree, cudaStream_t stream);
void launch_step_finalize_agreed(const StepPartial* partials, int nblocks, DevBudget* budget, Status* st,
                                 const long long* agreed, cudaStream_t stream);
// Copies up to kCopySegs strided runs of doubles (rows x n, 16-byte aligned
// addresses and counts of whole double pairs) in one launch; destinations may
// be another GPU's memory (peer access enabled): the halo exchange of the
// slab form. Skipped when st->failed is set (st may be null).
constexpr int kCopySegs = 24;
struct CopySeg {
    const double* src;
    double* dst;
    long long n, rows, src_pitch, dst_pitch;   // doubles
};
struct CopyList {
    CopySeg s[kCopySegs];
    int count, pad;
};
void launch_copy_segments(const CopyList& L, const Status* st, cudaStream_t stream);
// Refresh for output: mu_O, mu_Cr, M_O, M_Cr at every cell (3S:597-620)
void launch_refresh(const StepParams& P, const double* o, const double* cr, const double* p,
                    const double* gb, double* muO, double* muCr, double* mo, double* mc,
                    cudaStream_t stream);

// Device self-check of the exact division: mismatches against IEEE a/b
long long check_division(double b, long long n, unsigned long long seed, long long* tested);

// ---- init --------------------------------------------------------------------
struct InitParams {
    Grid g;
    int ng;
    double nxd, nyd, nzd;        // grid extents as doubles (periods)
    double bulk_cr, layer_o;
    int inlet_layer;             // bc == concentration
    // X slab: stored plane 0 is domain plane x_off; sums and counts cover the
    // own planes [x_lo, x_hi) only. A whole domain: 0, 0, g.nx.
    int x_off, x_lo, x_hi;
};
void launch_init_fields(const InitParams& I, double* o, double* cr, double* p, cudaStream_t stream);
// 3D Voronoi labels (first nearest seed under minimum image) and the distance
// to the nearest bisector (3S:450-466). seeds: x,y,z per seed. competitor
// (may be null) receives the 0-based seed of the nearest bisector (-1: none).
void launch_voronoi3(const InitParams& I, const double* seeds, double* grain, double* db,
                     int* volumes, int* competitor, cudaStream_t stream);
// Face adjacency of the grains (ng x ng bytes, set to 1 for adjacent pairs)
void launch_grain_adjacency(const InitParams& I, const double* grain, unsigned char* adj, cudaStream_t stream);
// 3D eta initial weights: per competitor g, the bisector distance (3S:469-494);
// the owner's slot receives -1. Output layout eta[g*nstore + idx].
void launch_eta_dist3(const InitParams& I, const double* seeds, const double* grain, double* eta,
                      cudaStream_t stream);
// Centre seed (3S:725-751): stamps the ball and accumulates nucO, nucCr, cells
void launch_center_seed(const InitParams& I, double cx, double cy, double cz, double r, int neta,
                        double* o, double* cr, double* p, double* eta, StepPartial* partials,
                        cudaStream_t stream, int* nblocks_out);
// Generic dd sum over the partial array (first nsum slots + count) into out
void launch_reduce_partials(const StepPartial* partials, int nblocks, StepPartial* out,
                            cudaStream_t stream);

// ---- diagnostics ---------------------------------------------------------------
// sums o, cr, p, h(p) (dd) and min/max of O, Cr, Ni, phi (3S:963-977)
struct DiagOut {
    double sum[4][2];
    double mn[4], mx[4];   // O, Cr, Ni(=1-o-cr, min only), phi
    long long mni[4], mxi[4];  // first cell (reference order) attaining each extremum
};
// grain_log statistics (3S:566-590): scalars, per-grain dominant cells and
// weighted amounts, and the discrete grain energy (3S:546-565)
struct GrainParams {
    Grid g;
    int dim, neta;
    double dx, da, db, K, W, A;
    const double* pairs;   // 2D: eta_pairs of the last mask (2D:337); unused in 3D
    int x_above;           // the plane after g's last one is stored and in the domain (an X slab
                           // below another): the last plane keeps its +X gradient term
};
struct GrainOut {
    double lo, hi, slo, shi, gbmax;
    double sum[3][2];      // S, (1-h) gb, energy
    long long unassigned;
};
struct GrainWork {
    unsigned long long* cells;  // neta
    void* parts;                // grain_blocks() * grain_part_bytes()
    double* amount_parts;       // grain_blocks() * neta * 2
};
size_t grain_part_bytes();
int grain_blocks(long long ncells);
void launch_grain_stats(const GrainParams& G, const double* eta, const double* s2, const double* p, const double* gb,
                        GrainWork& W, GrainOut* out, double* amount_out, long long* cells_out, cudaStream_t stream);

void launch_diagnostics(const Grid& g, const double* o, const double* cr, const double* p,
                        DiagOut* partials, int* nblocks, DiagOut* out, cudaStream_t stream);

}  // namespace nicr
