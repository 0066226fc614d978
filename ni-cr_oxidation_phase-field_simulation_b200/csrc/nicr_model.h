// Host-side model: the B200 counterpart of the reference's class Model
// (3S:336-978, 2D:194-711). It owns one domain resident in device memory and
// orchestrates the kernels; host code does only what must match the C library
// bit for bit at initialisation (random seeds via libstdc++, exp/hypot of the
// Voronoi mask and eta weights) and the formatting of output files.
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_kernels.h"
#include "nicr_ksp.h"
#include "nicr_physics.h"

namespace nicr {

// Error carrying a nicr status code; the message is the reference's text.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char* what);
// The message nicr_last_error(NULL) returns after a failed creation.
void set_create_error(const std::string& e);

// An X slab of a larger 3D domain (the slab form, nicr_slabs.cpp): the model
// owns domain planes [x0, x1) and stores them with up to `halo` neighbour
// planes below and above (clipped to the domain), which its group refreshes
// from the neighbouring slabs; every stored plane is initialised like the
// whole domain's, so the halos start consistent.
struct SlabSpec {
    int x0 = 0, x1 = 0, halo = 0;
};
class SlabGroup;
class SlabRank;

// Colours ng grains with k colours from their face adjacency (adj: ng x ng
// bytes): DSatur order (most distinct neighbour colours, then most
// neighbours, then lowest index), each grain taking the lowest colour no
// coloured neighbour has, or when all k are taken the colour fewest coloured
// neighbours have (lowest first). Deterministic; returns one colour per grain.
std::vector<int> colour_grains(const std::vector<unsigned char>& adj, int ng, int k);
int run_self_test(int dim);   // --self-test (nicr_selftest.cpp)

class Model {
public:
    explicit Model(const nicr_config& cfg, const SlabSpec* slab = nullptr);
    ~Model();
    Model(const Model&) = delete;
    Model& operator=(const Model&) = delete;

    nicr_config c;
    Grid g{};
    int dim;
    bool has_eta = false;      // grain_evolution && grains (3S:343)
    bool advance_eta = false;  // eta trial/swap each step (3S:810, 2D:591)
    int neta = 0;
    EtaCoef ec{};
    std::vector<double> seeds;         // dim doubles per seed
    std::vector<long long> volumes;
    int center_seed_cells = 0;
    bool grain_retained = true;        // 3D frees the id map when eta is active (3S:377-380)
    double next_nucleation;
    long long steps_done = 0;          // accepted steps (host view)
    std::string last_error;
    // slab form: stored plane 0 is domain plane x_off; own planes [sp.x_lo, sp.x_hi)
    bool is_slab = false;
    int x_off = 0;

    cudaStream_t stream = nullptr;
    bool owns_stream = true;
    // Output machinery that outlives single calls (the asynchronous VTI
    // writer of nicr_output.cpp); released, after its pending writes, first
    // thing in the destructor.
    std::shared_ptr<void> output_writer;
    // Use stream s (owned by the caller, e.g. a batch) for all further work.
    void adopt_stream(cudaStream_t s);

    // ---- API used by the C-ABI
    void set_field(int field, int index, const double* host);
    void get_field(int field, int index, double* host);
    void refresh();                    // materialise mu/M (and eta mask) for output
    void invalidate_eta_cache() { eta_dirty = true; }
    void reset_inventory();
    int step(int nsteps, int* completed);            // Model::step x n
    int run(int nsteps, int* completed);             // run() schedule
    int nucleate(int* nuclei);
    int stamp(int x, int y, int z, int* cells);
    void budget(nicr_budget* b);
    void diagnostics(nicr_diagnostics* d);
    void grain_stats(nicr_grain_stats* s, long long* cells, double* amount);
    size_t device_bytes() const { return dev_bytes; }
    // checkpoint / restart (nicr_checkpoint.cpp)
    void save_state(const std::string& path);
    void load_state(const std::string& path);
    void sync();

    // measurement hooks: CUDA events around every kernel launch (when enabled)
    // and a count of the kernels this model launched
    enum Kern { K_STEP_MAIN, K_ETA_UPDATE, K_FINALIZE, K_ETA_MASK, K_KSP, K_REFRESH, K_DIAG, K_STEP_ETA,
                K_STEP_FUSED, K_COUNT };
    static const char* kernel_name(int k);
    void profile_enable(bool on);
    void profile_collect();
    double prof_ms[K_COUNT] = {};
    long long prof_n[K_COUNT] = {};
    long long launches = 0;

    // One step split into phases, for batches that launch the step kernel of
    // many domains at once: prepare_step (eta mask when stale), step_desc (the
    // step kernel's parameters and buffers), then complete_step (eta update,
    // optional finalize, buffer parity). run_begin / run_pre_step / run_end are
    // run()'s schedule (Ksp scans) and commit around those steps.
    struct RunPlan {
        long long before = 0;
        int nsteps = 0;
        bool schedule = false;
        double next = 0.;
        std::vector<double> sched;
    };
    // Planes per CTA of this domain's step and eta kernels (a batch sets one
    // chunk for all its domains). Grows the partial-sum buffer when needed.
    void set_xchunk(int c);
    // Times `reps` launches of this domain's step (and eta update) kernels for
    // each X chunk candidate and, in 3D, each occupancy variant, on the current
    // state without committing anything, and keeps the fastest pair.
    void tune(int reps, int* xchunk, int* minb);
    // One pass of the step kernels into the trial buffers (no commit), and of
    // the eta update alone.
    void launch_trial_kernels();
    void launch_trial_eta();
    void prepare_step();
    BatchDomain step_desc() const;
    FinalizeDomain finalize_desc(int nblocks) const;
    void complete_step(int nblocks, bool finalize);
    // step-pair graphs: whether they are used, whether step s of plan r
    // starts with a Ksp scan, and the buffer parity a captured pair keys on
    bool graphs_enabled() const;
    bool ksp_due(const RunPlan& r, int s) const;
    int parity_key() const { return cur | (ecur << 1) | (gcur << 2); }
    void run_begin(RunPlan& r, int nsteps, bool schedule);
    void run_pre_step(RunPlan& r, int s);
    int run_end(RunPlan& r, int* completed);

    // The own planes as a grid of their own (a whole domain: g) and their
    // offset in the stored arrays, for reductions over owned cells.
    Grid own_grid() const;
    long long own_offset() const { return (long long)sp.x_lo * g.plane; }
    InitParams init_params() const;
    // Device array of a field for reading (materialising mu/M, the mask or the
    // eta cache first), and of a state field for writing.
    const double* field_ptr(int field, int index);
    double* state_ptr(int field, int index);
    // Host copies of stored planes [x_begin, x_begin + count) of device array d.
    void copy_planes_out(const double* d, double* host, int x_begin, int count);
    void copy_planes_in(double* d, const double* host, int x_begin, int count);

    // raw device pointers of the current state (for tests, bench, writers)
    double* d_o() const { return o_[cur]; }
    double* d_cr() const { return cr_[cur]; }
    double* d_p() const { return p_[cur]; }
    double* d_gb() const { return gb_[gcur]; }
    double* d_eta(int gi) const { return eta_[ecur] + (size_t)gi * g.nstore; }
    double* d_grain() const { return grain; }
    StepParams params() const { return sp; }
    // device buffers the writers read (after refresh())
    const double* d_mu_o() const { return muO; }
    const double* d_mu_cr() const { return muCr; }
    const double* d_m_o() const { return mo; }
    const double* d_m_cr() const { return mc; }
    void fetch(const double* d, double* host) { copy_out(d, host); }
    void ensure_mask() { if (has_eta && (eta_dirty || dim == 2)) eta_mask_now(); }

    // One process per slab (nicr_slab_* in nicr_slab_rank.cpp): the step
    // kernels plus this step's signed agreement word (d_agree(), which the
    // ranks reduce with a MIN collective), then the commit that reads the
    // reduced word and flips parity.
    void rank_launch();
    void rank_commit();
    long long* d_agree();
    RunPlan rank_plan;

    // the step kernel and the eta update of a step as one launch (k_step_eta:
    // reciprocal form, 3D, 1..16 evolving eta fields; opt-in, NICR_FUSED=1:
    // measured 1.122 vs 1.129 ms per step at 256^3 with 8 fields)
    bool fused_step() const;
    // One HBM pass per step (k_step_fused: 3D, 1..8 evolving eta fields, rows
    // a multiple of 16, columns of 32) where nicr_config.step_form asks for it
    // (AUTO: the reciprocal form only); NICR_STEP_FORM=onepass|split overrides
    // every handle (A/B runs).
    // The pass rebuilds S and gb from eta on chip and writes neither, so the
    // handle's gb / eta_s2 arrays go stale (eta_dirty) and are rebuilt when read.
    bool onepass_step() const;
    bool onepass_failed = false;   // the launcher refused (buffer alignment): split form from then on
    // one step in the one-pass form into the trial buffers; false when it cannot launch
    bool launch_onepass(int* nb);

private:
    friend class SlabGroup;
    friend class SlabRank;
    unsigned* ticket = nullptr;
    int rank_nb = 0;
    long long* agree = nullptr;
    // slab form: the step kernels of one step into the trial buffers (no
    // commit; returns the step kernel's partial count), and the commit that
    // agrees with the other slabs on the step's outcome, then flips parity
    int slab_launch();
    void slab_commit(int nblocks, const SlabPeers& peers);
    StepParams sp{};
    size_t dev_bytes = 0;
    // state (ping-pong)
    double* o_[2] = {nullptr, nullptr};
    double* cr_[2] = {nullptr, nullptr};
    double* p_[2] = {nullptr, nullptr};
    int cur = 0;
    double* gb_[2] = {nullptr, nullptr};   // mask; [1] used only when eta advances
    double* s2_[2] = {nullptr, nullptr};
    int gcur = 0;
    double* eta_[2] = {nullptr, nullptr};  // neta fields each
    int ecur = 0;
    double* grain = nullptr;
    double* pairs = nullptr;               // 2D eta_pairs (output only)
    double* gb_initial = nullptr;          // 2D gb_initial (output only)
    double *muO = nullptr, *muCr = nullptr, *mo = nullptr, *mc = nullptr;
    bool eta_dirty = true;
    // reductions / status
    StepPartial* partials = nullptr;
    int partial_cap = 0;
    Status* st = nullptr;
    DevBudget* bud = nullptr;
    DiagOut* diag_part = nullptr;
    DiagOut* diag_out = nullptr;
    StepPartial* red_out = nullptr;
    // Ksp
    KspDev kd{};
    KspWork kw{};
    KspResult* kres = nullptr;
    int* d_shadow = nullptr;
    int* d_ball = nullptr;
    unsigned char* d_hyp = nullptr;
    // grain statistics work buffers (allocated on first use)
    GrainWork gw{};
    GrainOut* g_out = nullptr;
    double* g_amount = nullptr;
    long long* g_cells = nullptr;
    // pinned host staging for small results
    Status* h_st = nullptr;
    // profiling
    bool prof_on = false;
    std::vector<cudaEvent_t> prof_pool;
    size_t prof_used = 0;
    struct Mark { int k; size_t e0; };
    std::vector<Mark> prof_marks;
    size_t prof_begin();
    void prof_end(int k, size_t e0, int kernels);

    // captured runs of 2, 4, 8 or 16 steps, one per length and starting
    // buffer parity (cur, ecur, gcur)
    struct PairGraph {
        cudaGraphExec_t exec = nullptr;
        int key = 0;
        long long kernels = 0;
    };
    PairGraph pair_graphs[32];
    void launch_step_group(int nsteps);
    int group_length(const RunPlan& r, int s, int nsteps) const;

    void release();
    double* dalloc(size_t n);
    template <class T> T* dalloc_t(size_t n);
    void voronoi();
    void voronoi2d_host(std::vector<double>& grain_h, std::vector<double>& gb_h);
    void init_center_seed();
    void init_eta();
    // eta_colours > 0: the grains' face adjacency over the stored cells, the
    // colour of each grain, and the eta fields from the colours (kept from
    // voronoi(): the nearest-bisector distance and competitor of every cell)
    void grain_adjacency();
    void alloc_eta(int n);
    void init_eta_coloured();
    std::vector<unsigned char> adjacency;
    std::vector<int> seed_colour;
    std::vector<double> init_db;
    std::vector<int> init_comp;
    void setup_ksp();
    void enqueue_step();
    void reset_status();
    int finish_batch(long long steps_before, int enqueued, const std::vector<double>* nuc_sched, int* completed);
    std::string describe_failure(unsigned long long key, int parity_next);
    void copy_out(const double* d, double* host);
    void copy_in(double* d, const double* host);
    void eta_mask_now();
};

}  // namespace nicr

// The opaque handle of include/nicr.h: one model and its last error message.
struct nicr_handle {
    nicr::Model* m = nullptr;
    std::string err;
    bool borrowed = false;   // a domain owned by a nicr_batch: nicr_destroy leaves it alone
};
