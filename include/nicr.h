/*
 * nicr.h — C-ABI of the B200 Ni–Cr oxidation phase-field solver.
 *
 * One opaque handle owns one simulation domain resident in GPU memory (all
 * fields, trial buffers, budgets). Host buffers passed in or out are owned by
 * the caller and copied. Every entry point returns an int status (NICR_OK or a
 * negative/positive code below); no C++ exception crosses this boundary. A
 * handle is bound to one CUDA device and one stream and is not thread-safe.
 *
 * The reference has no FFI: its in-process surface is the C++ class `Model`
 * that its test drivers reach with `#define main ...; #include` (reference
 * mpi3d-slab/tests/regression_driver.cpp:1-8). Each entry point below names the
 * Model member it replaces (2D = mpi2d/NiCr2D_grains.cpp,
 * 3S = mpi3d-slab/NiCr3D_grains.cpp). Field data are exchanged in the
 * reference's interior order: X slowest, Z fastest in 3D (3S:165-167); X
 * slowest, Y fastest in 2D (2D:149); ghost layers are never exchanged.
 */
#ifndef NICR_H
#define NICR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replacing std::runtime_error, 3S:117-127) ---------------- */
enum {
    NICR_OK = 0,
    NICR_ERR_INVALID_ARG = 1,       /* bad parameter / bounds (parse 3S:1055-1081) */
    NICR_ERR_TRIAL_NONFINITE = 2,   /* "Nonfinite trial field" (3S:790)            */
    NICR_ERR_TRIAL_BOUNDS = 3,      /* "Out-of-bounds trial at" (3S:799-804)       */
    NICR_ERR_ETA_RANGE = 4,         /* "Eta trial outside [0,1]" (3S:518-523)      */
    NICR_ERR_CUDA = 5,              /* CUDA runtime failure                         */
    NICR_ERR_NO_DEVICE = 6,         /* no usable CUDA device / extension missing    */
    NICR_ERR_STATE = 7,             /* call not valid in the handle's state         */
    NICR_ERR_IO = 8                 /* output file could not be written             */
};

/* ---- enumerations of the reference's string options (3S:56-58) ------------- */
enum { NICR_BC_CONCENTRATION = 0, NICR_BC_MU = 1, NICR_BC_CLOSED = 2 };
enum { NICR_CK_LEGACY = 0, NICR_CK_OFF = 1 };
enum { NICR_BOUNDS_STOP = 0, NICR_BOUNDS_LEGACY = 1 };
enum { NICR_NUC_KSP = 0, NICR_NUC_CENTER = 1, NICR_NUC_OFF = 2 };
/* Arithmetic form. NICR_FP64 is the drop-in: the same IEEE operations in the
 * same order as the reference, so single-process results are bit-identical.
 * NICR_FP64_FAST keeps the FP64 state and operation order but multiplies by
 * RN(1/b) where the reference divides by a run constant b (dx^2, dx, dt),
 * each such quotient within one ulp; its deviation from NICR_FP64 is tested
 * and reported by the benchmark. No counterpart in the reference.             */
enum { NICR_FP64 = 0, NICR_FP64_FAST = 1 };

/* ---- configuration: struct Config + struct Physics (3S:43-79, 2D:39-71) ---- */
typedef struct nicr_config {
    int dim;                      /* 2 (mpi2d) or 3 (mpi3d-slab)                */
    int nx, ny, nz;               /* cells; nz ignored when dim == 2            */
    int steps, output_every;      /* run-loop controls (CLI level)              */
    int left_edge_sites;          /* --left-edge-sites / --left-face-sites      */
    int max_eta_fields;           /* --max-eta-fields                           */
    unsigned long long random_seed;
    double dx, dy, dz, dt;
    double grain_diameter_grid, gb_fwhm_grid;
    double gb_factor_o, gb_factor_cr;
    double radius_grid, exclusion_gap_grid, nucleation_period;
    double mu_res, surface_c_ref;
    int bc, ck, bounds, nucleation;   /* NICR_BC_*, NICR_CK_*, NICR_BOUNDS_*, NICR_NUC_* */
    int grains, oxygen_diffusion, grain_evolution, frozen_eta_cache;
    double eta_W, eta_kappa, eta_L, eta_oxide_penalty;
    int eta_output_all;           /* --eta-output all (1) | summary (0)         */
    int output_vti;               /* 3D --output-format vti (1) | vtk (0)       */
    int output_float64;           /* 3D --output-precision float64 (1) | float32 */
    int compression_level;        /* 3D --compression-level 0..9                */
    /* Physics constants that the reference fixes as constexpr (3S:73-79). The
     * defaults reproduce it; a parameter sweep may change them per run.       */
    double ksp;                   /* Physics::ksp    = 1.28e-7                  */
    double bulk_cr;               /* Physics::bulkCr = 0.1986                   */
    double layer_o;               /* Physics::layerO = 0.0023                   */
    int precision;                /* NICR_FP64 (drop-in) or NICR_FP64_FAST      */
    int device;                   /* CUDA device ordinal                        */
    int checkpoint_every;         /* programs: write out/checkpoint.bin every N
                                     steps (0: never); no reference counterpart */
    int eta_colours;              /* 3D evolving grains: 0 = one eta per Voronoi
                                     grain (the reference, 3S:469-494); K > 0 =
                                     the grains coloured into K eta fields, no
                                     two face-adjacent grains sharing one where
                                     K colours allow, with tanh profiles across
                                     the boundaries; no reference counterpart */
    int step_form;                /* 3D evolving grains (no reference
                                     counterpart): NICR_STEP_AUTO, NICR_STEP_ONEPASS
                                     (one HBM pass: the step and the eta update in
                                     one kernel, where the grid allows it) or
                                     NICR_STEP_SPLIT (two kernels); the fields are
                                     the same bit for bit in the drop-in form */
    int reserved[3];
} nicr_config;

/* nicr_config.step_form. AUTO takes the one-pass kernel wherever the grid
 * allows it (the faster form in both arithmetic forms on B200) and the two
 * kernels elsewhere; the environment variable NICR_STEP_FORM=onepass|split
 * overrides every handle of the process (benchmarks). */
enum { NICR_STEP_AUTO = 0, NICR_STEP_ONEPASS = 1, NICR_STEP_SPLIT = 2 };

/* Fills the reference defaults for dim 2 or 3 (Config{} at 2D:39 / 3S:43). */
void nicr_config_default(nicr_config* cfg, int dim);

/* Parses the reference's command-line flags into cfg (parse, 2D:718-790 /
 * 3S:986-1082), with the same validation and messages. Returns NICR_OK,
 * NICR_ERR_INVALID_ARG (message in err), or 100 for --help/--version (text in
 * err). out_dir receives --out; self_test receives --self-test.               */
int nicr_config_parse(nicr_config* cfg, int dim, int argc, const char* const* argv,
                      char* out_dir, size_t out_dir_len, int* self_test,
                      char* err, size_t err_len);

/* ---- fields --------------------------------------------------------------- */
enum {
    NICR_FIELD_O = 0,        /* Model::o              */
    NICR_FIELD_CR = 1,       /* Model::cr             */
    NICR_FIELD_PHI = 2,      /* Model::p              */
    NICR_FIELD_ETA = 3,      /* Model::eta[index]     */
    NICR_FIELD_MU_O = 4,     /* Model::muO  (refreshed when read)           */
    NICR_FIELD_MU_CR = 5,    /* Model::muCr (refreshed when read)           */
    NICR_FIELD_M_O = 6,      /* Model::mo   (refreshed when read)           */
    NICR_FIELD_M_CR = 7,     /* Model::mc   (refreshed when read)           */
    NICR_FIELD_GB = 8,       /* Model::gb  (Voronoi mask or eta-derived)    */
    NICR_FIELD_GRAIN = 9,    /* Model::grain (initial Voronoi id, 1-based)  */
    NICR_FIELD_ETA_S2 = 10,  /* Model::eta_s2                               */
    NICR_FIELD_ETA_PAIRS = 11, /* 2D Model::eta_pairs                       */
    NICR_FIELD_GB_INITIAL = 12 /* 2D Model::gb_initial                      */
};

typedef struct nicr_handle nicr_handle;

/* Model::Model(Config, MPI_COMM_SELF) (2D:208-228, 3S:356-384): allocates the
 * domain on the GPU, builds the Voronoi grains, initial fields, centre seed and
 * eta fields, and refreshes. */
int nicr_create(const nicr_config* cfg, nicr_handle** out);
void nicr_destroy(nicr_handle* h);
/* Message of the last failure on this handle, in the reference's wording. */
const char* nicr_last_error(const nicr_handle* h);

typedef struct nicr_info {
    int dim, nx, ny, nz;
    int n_seeds;              /* seeds.size()                                 */
    int n_eta;                /* eta.size()                                   */
    int center_seed_cells;    /* Model::center_seed_cells                     */
    int grain_map_retained;   /* 3D frees the initial id map when eta is active */
    long long n_cells;
    long long steps_done;     /* accepted steps since creation                */
    size_t device_bytes;      /* device memory held by the handle             */
} nicr_info;
int nicr_get_info(const nicr_handle* h, nicr_info* info);

/* Seeds (x,y[,z] per seed, grid units) and per-grain cell counts (3S:395-467). */
int nicr_get_seeds(const nicr_handle* h, double* xyz, long long* volumes);

/* Copies one field between host memory and the device (interior cells only,
 * reference order). Setting O/CR/PHI/ETA also invalidates the frozen-eta
 * cache, as the reference drivers do after editing fields (3S:1092-1101
 * fill_smooth; 3S:347-349 invalidate_eta_cache); the eta mask and mu/M are
 * recomputed when next needed (the next step, or reading GB, ETA_S2, MU_*,
 * M_*). Host buffers in pinned memory transfer at full PCIe speed. */
int nicr_set_field(nicr_handle* h, int field, int index, const double* host);
int nicr_get_field(nicr_handle* h, int field, int index, double* host);
/* Device view of one field of the current state (no copy; no counterpart in
 * the reference): *ptr points at cell (0, 0, 0) and cell (i, j, k) of the
 * nx x ny x nz grid (2D: nx x 1 x ny) is (*ptr)[(i * ny + j) * pitch + k],
 * FP64. The view is valid until the next step, nucleation, load or field
 * write of the handle (steps alternate buffers); the handle's stream has no
 * work pending when it returns. writable = 1 (O, CR, PHI, ETA only) marks
 * the frozen-eta cache stale as nicr_set_field does; the caller then writes
 * through the view before the next call on the handle, on a stream ordered
 * with the handle's (nicr_stream). Whole-domain handles only. */
int nicr_field_device(nicr_handle* h, int field, int index, int writable, void** ptr, long long* pitch);

/* Model::refresh (3S:597-620): materialises mu_O, mu_Cr, M_O, M_Cr (and the
 * eta mask) for output. Steps do not need it; they fuse it on chip. */
int nicr_refresh(nicr_handle* h);
/* Model::invalidate_eta_cache (3S:349). */
int nicr_invalidate_eta_cache(nicr_handle* h);
/* initialO = sum(o), initialCr = sum(cr) (3S:370): used by drivers that inject
 * fields after construction. */
int nicr_reset_inventory(nicr_handle* h);

/* Model::step x nsteps (3S:761-826, 2D:551-597). Stops at the first rejected
 * trial: *completed = accepted steps; the state is the last accepted one, the
 * budget is restored (3S:812-820) and the status names the failure. Pairs of
 * steps are replayed as captured CUDA graphs (results identical to launching
 * each kernel; NICR_GRAPHS=0 in the environment launches them one by one). */
int nicr_step(nicr_handle* h, int nsteps, int* completed);
/* nsteps of run()'s loop (3S:1368-1385, 2D:1219-1236): before each step, Ksp
 * nucleation when its physical time is due, then Model::step. The schedule
 * continues across calls. */
int nicr_run(nicr_handle* h, int nsteps, int* completed);
/* Model::nucleate (3S:752-759): ordered Ksp scan and hard-seed insertion.   */
int nicr_nucleate(nicr_handle* h, int* stamped_nuclei);
/* Model::stamp (3S:704-724); z ignored in 2D. *cells = voxels changed.       */
int nicr_stamp(nicr_handle* h, int x, int y, int z, int* cells);

/* struct Budget (3S:217). The reference accumulates in long double; each sum
 * is returned as an unevaluated pair hi+lo of doubles (hi = rounded value).  */
typedef struct nicr_budget {
    double nucO[2], nucCr[2], ckO[2], ckCr[2], clipO[2], clipCr[2], bcO[2], bcCr[2];
    long long nuclei, clipped;
    double initialO[2], initialCr[2];
} nicr_budget;
int nicr_get_budget(const nicr_handle* h, nicr_budget* b);

/* Values of one diagnostics.csv row (Model::log, 3S:963-977 / 2D:697-710). */
typedef struct nicr_diagnostics {
    double sum_O[2], sum_Cr[2], sum_phi[2], sum_h[2];
    double min_O, max_O, min_Cr, max_Cr, min_Ni, min_phi, max_phi;
} nicr_diagnostics;
int nicr_get_diagnostics(nicr_handle* h, nicr_diagnostics* d);

/* Values of one grain_diagnostics.csv row and the per-grain history
 * (Model::grain_log, 3S:566-590 / 2D:382-406). Arrays hold n_eta entries.   */
typedef struct nicr_grain_stats {
    double min_eta, max_eta, min_s2, max_s2;
    double sum_s2[2], mask[2], energy[2];
    double gb_max;
    long long alive, unassigned;
} nicr_grain_stats;
int nicr_get_grain_stats(nicr_handle* h, nicr_grain_stats* s, long long* cells, double* amount_hi_lo);

/* Output writers (host C++ over device data): the reference's files, byte for
 * byte where the values are bit-identical. */
int nicr_write_vtk(nicr_handle* h, const char* path);          /* 2D:598-632, 3S:828-856 */
int nicr_write_vti(nicr_handle* h, const char* path);          /* 3S:857-869, 238-334    */
/* Asynchronous VTI frame (the reference writes synchronously, 3S:238-334).
 * nicr_write_vti_async enqueues on the handle's stream the frame's arrays,
 * built on the GPU in file order and type, and their copy to pinned host
 * memory, then returns; a library thread compresses (64 KiB zlib blocks, in
 * parallel) and writes the file while the caller keeps stepping. The file is
 * byte-identical to nicr_write_vti's of the same state. One frame is in
 * flight per handle: the next nicr_write_vti(_async) or nicr_output_wait
 * first completes it and returns its error, if any (NICR_ERR_IO with the
 * reference's message). nicr_destroy completes it too. */
int nicr_write_vti_async(nicr_handle* h, const char* path);
int nicr_output_wait(nicr_handle* h);
int nicr_write_metadata(nicr_handle* h, const char* out_dir);  /* 2D:633-696, 3S:874-962 */
/* Formats one diagnostics.csv row / grain rows for step n into buf.          */
int nicr_format_log_row(nicr_handle* h, int n, char* buf, size_t len);
int nicr_format_grain_rows(nicr_handle* h, int n, char* diag, size_t diag_len,
                           char* history, size_t history_len);

/* One step of c_O, c_Cr and phi on caller-owned device memory, for callers
 * that must not allocate device memory (a coupling code that owns all of HBM
 * through its own pool, or code running where the CUDA memory API may not be
 * called). No counterpart in the reference, which has no GPU.
 *
 * The arithmetic form is cfg->precision: NICR_FP64 (the drop-in form,
 * bit-identical to the reference) or NICR_FP64_FAST (the reciprocal form);
 * any other value returns NICR_ERR_INVALID_ARG, as nicr_create does.
 *
 * It allocates nothing: o, cr, p (inputs) and o_next, cr_next, p_next
 * (outputs) are packed device arrays in interior order (X slowest, column
 * pitch nz in 3D and ny in 2D); gb is the grain-boundary mask when grains are
 * on, eta_s2 the sum of eta^2 when eta evolves. The step's scratch lives in a
 * file-scope device array of the library (about 768 KB per GPU, held until
 * exit) that holds the partial sums of at most 8192 CTAs of the step kernel.
 * The call lengthens the X chunk (planes per CTA) until the grid fits, so it
 * serves every grid with at most 8192 step tiles per X plane (3D:
 * ceil(ny/8)*ceil(nz/32) <= 8192; 2D: ceil(ny/128) <= 8192); larger grids
 * return NICR_ERR_INVALID_ARG before touching the device. The fields do not
 * depend on the chunk; the budget increments may differ from the handle
 * API's in the last bits (~1e-16 relative). The first call on a device
 * resolves the array's device address, so make it before any stream capture.
 * Every call shares the array and clears its status word first; calls that
 * overlap on the GPU race on it. If a CUDA error is already pending on the
 * calling thread, the call enqueues nothing, leaves that error in place and
 * returns NICR_ERR_CUDA; otherwise it reads and clears only the launch errors
 * of its own kernels. The kernels are enqueued on `stream` (a cudaStream_t,
 * NULL for the legacy default stream) and write *result (device memory)
 * asynchronously: trial_key == ~0 when every trial was accepted; otherwise
 * the trial buffers hold a rejected step (key/4 = first failing cell in
 * reference order, key%4: 0 nonfinite, 1 out of bounds) and must not be
 * swapped in. */
typedef struct nicr_step_result {
    double ckO[2], ckCr[2], clipO[2], clipCr[2], bcO[2];  /* budget increments (hi, lo) */
    long long clipped;                                     /* cells clipped this step     */
    unsigned long long trial_key;                          /* ~0 = accepted               */
} nicr_step_result;
int nicr_step_noalloc(const nicr_config* cfg, const double* o, const double* cr, const double* p,
                      const double* gb, const double* eta_s2, double* o_next, double* cr_next,
                      double* p_next, nicr_step_result* result, void* stream);

/* Autotuning (no counterpart in the reference). nicr_tune times `reps`
 * passes of the step kernels (and the eta update) on the handle's current
 * state for every X chunk the chooser considers (planes per CTA) and, in 3D,
 * both occupancy variants of the step kernel, writing only trial buffers, and
 * keeps the fastest; the state, budget and step count are unchanged. Fields
 * of later steps are the same bit for bit whatever is chosen; budget sums,
 * reduced per CTA, may differ in the last digits (~1e-16 relative).
 * nicr_batch_tune chooses the batch's common X chunk the same way. The choice
 * is returned in *xchunk / *minb when not NULL. */
typedef struct nicr_batch nicr_batch;
int nicr_tune(nicr_handle* h, int reps, int* xchunk, int* minb);
int nicr_batch_tune(nicr_batch* b, int reps, int* xchunk);

/* Checkpoint / restart (no counterpart in the reference, which cannot resume
 * a run). nicr_save_state writes the handle's state to `path`: a header (the
 * configuration, accepted steps, nucleation clock, budget, Voronoi seeds),
 * then the refreshed interior fields o, cr, p, muO, muCr, mo, mc, gb,
 * [eta_s2], eta_1..N in the order and layout of the reference's
 * snapshot_state dump (mpi3d-slab/tests/regression_driver.cpp:17-32: X
 * slowest, Z fastest, FP64), then the grain map when kept and the 2D initial
 * GB mask, and a checksum. nicr_load_state restores such a file into a handle
 * created from the same configuration (run length, output options, device and
 * arithmetic form may differ; any other difference is NICR_ERR_INVALID_ARG
 * naming the field), after which stepping continues bit for bit as the
 * uninterrupted run would. A truncated or corrupted file is rejected before
 * the handle is touched. */
int nicr_save_state(nicr_handle* h, const char* path);
int nicr_load_state(nicr_handle* h, const char* path);

/* Batched multi-domain form: n independent domains on one device (all
 * cfgs[i].device equal), e.g. a parameter sweep of many small grids. Each
 * domain is created exactly as nicr_create(&cfgs[i]) would create it and
 * evolves as its own handle would: the same kernels give bit-identical
 * fields; the batch gives all its domains one X chunk (planes per CTA, chosen
 * for their total CTA count), so budget sums, reduced per CTA, agree with a
 * lone handle's to ~1e-16 relative rather than bit for bit. The batch changes
 * the launch structure of a step: one step launch per group of up to 48
 * consecutive domains of one dimensionality and precision, one commit launch
 * for all domains, all on the batch's stream. The
 * reference runs one domain per program (3S:1309-1395); there is no
 * counterpart of the batch itself.
 *
 * nicr_batch_domain returns a borrowed handle of domain i for every per-domain
 * call of this header (fields, budgets, diagnostics, writers, nucleate,
 * stamp); nicr_destroy ignores it, nicr_batch_destroy frees it. Running a
 * borrowed handle on its own (nicr_step/nicr_run) is allowed and uses the
 * batch's stream. nicr_batch_step advances every domain nsteps steps
 * (Model::step), nicr_batch_run follows each domain's run() schedule (Ksp
 * scans); completed[i] (n entries, may be NULL) receives the accepted steps of
 * domain i. A domain whose trial fails stops at its last accepted state, as
 * nicr_run leaves a handle, while the others complete; the return value is
 * the status of the first failing domain (NICR_OK when none failed) and
 * nicr_batch_last_error names it ("domain i: <message>"). */
int nicr_batch_create(const nicr_config* cfgs, int n, nicr_batch** out);
void nicr_batch_destroy(nicr_batch* b);
int nicr_batch_size(const nicr_batch* b);
nicr_handle* nicr_batch_domain(nicr_batch* b, int i);
int nicr_batch_step(nicr_batch* b, int nsteps, int* completed);
int nicr_batch_run(nicr_batch* b, int nsteps, int* completed);
const char* nicr_batch_last_error(const nicr_batch* b);
long long nicr_batch_kernel_launches(const nicr_batch* b);
void* nicr_batch_stream(const nicr_batch* b);

/* Slab form: one 3D domain split along X into nslabs slabs of near-equal
 * plane counts, slab i on GPU devices[i] (devices may repeat; NULL puts every
 * slab on cfg->device). This is mpi3d-slab's own decomposition (each MPI rank
 * owns a range of X planes and trades ghost planes with its neighbours,
 * 3S:146-191, MPI_Allreduce of the budget, root-gathered Ksp scan 3S:666-686),
 * with GPUs in place of ranks: each slab stores its planes plus `halo` planes
 * of each neighbour (2, or ceil(radius + gap) with Ksp nucleation), refreshed
 * after every step by a copy kernel that stores into the neighbour's memory
 * (P2P over NVLink between GPUs); the slabs agree on each step's acceptance
 * on the device, and Ksp scans resolve slab after slab in X order. Fields
 * are bit-identical to a single handle's on the same configuration in the
 * drop-in form (in the reciprocal form, where the slab kernels are compiled
 * with FMA contraction apart from the whole-domain ones, to rounding: 1e-13
 * relative); budget sums (per-slab double-double sums added) agree to ~1e-16
 * relative. Every
 * slab needs at least `halo` planes; peer access must be possible between all
 * devices used. nicr_slabs_step / _run follow nicr_step / nicr_run
 * (failures: all slabs stop at the last accepted state, the message names the
 * failing cell as nicr_last_error would). Fields are exchanged whole-domain
 * (X slowest, like nicr_get_field). No 2D form. */
typedef struct nicr_slabs nicr_slabs;
int nicr_slabs_create(const nicr_config* cfg, int nslabs, const int* devices, nicr_slabs** out);
void nicr_slabs_destroy(nicr_slabs* s);
int nicr_slabs_count(const nicr_slabs* s);
int nicr_slabs_n_eta(const nicr_slabs* s);      /* eta fields of the domain */
/* domain planes [*x0, *x1) of slab i, its device and the halo width */
int nicr_slabs_info(const nicr_slabs* s, int i, int* x0, int* x1, int* device, int* halo);
int nicr_slabs_step(nicr_slabs* s, int nsteps, int* completed);
int nicr_slabs_run(nicr_slabs* s, int nsteps, int* completed);
int nicr_slabs_nucleate(nicr_slabs* s, int* nuclei);
int nicr_slabs_get_field(nicr_slabs* s, int field, int index, double* host);
int nicr_slabs_set_field(nicr_slabs* s, int field, int index, const double* host);
int nicr_slabs_reset_inventory(nicr_slabs* s);
int nicr_slabs_get_budget(nicr_slabs* s, nicr_budget* b);
int nicr_slabs_get_diagnostics(nicr_slabs* s, nicr_diagnostics* d);
/* nicr_get_grain_stats over the whole domain (cells, amount: n_eta entries) */
int nicr_slabs_get_grain_stats(nicr_slabs* s, nicr_grain_stats* st, long long* cells, double* amount);
/* nicr_write_vti of the whole domain: the same file a single handle writes */
int nicr_slabs_write_vti(nicr_slabs* s, const char* path);
long long nicr_slabs_steps_done(const nicr_slabs* s);
long long nicr_slabs_kernel_launches(const nicr_slabs* s);
/* stream (a cudaStream_t) slab i enqueues on */
void* nicr_slabs_stream(const nicr_slabs* s, int i);
const char* nicr_slabs_last_error(const nicr_slabs* s);

/* Slab form with one process per GPU: a handle holding slab `index` of the
 * domain split along X into nslabs slabs (the partition and halo width of
 * nicr_slabs_create), initialised like the whole domain's planes. The caller
 * communicates between the ranks (the python package's slab_ranks module does
 * it over torch.distributed with NCCL), per step:
 *   nicr_slab_launch    the step kernels, then this step's agreement word
 *                       (nicr_slab_agree_word: an int64 on the device,
 *                       INT64_MAX when every trial passed, else the failing
 *                       cell's key in whole-domain order)
 *   MIN all-reduce of the agreement words over the ranks, in place
 *   nicr_slab_commit    commit with the reduced word (all ranks accept or
 *                       reject alike), flip the buffer parity
 *   halo exchange: each rank sends nicr_slab_region(which = 0 / 1) planes
 *   to the rank below / above and receives into which = 2 / 3: o and cr two
 *   planes deep, phi one, and with evolving grains gb and every eta one.
 * Batches of steps: nicr_slab_begin(n, schedule), per step s
 * nicr_slab_scan_due(s) (a Ksp scan is due before step s: exchange phi
 * `halo` planes deep, nicr_slab_scan_candidates on every rank, then
 * nicr_slab_scan_resolve rank after rank in X order with the nuclei the
 * lower ranks accepted in this scan as `pre` (KspNucleus: x, y, z, full;
 * nicr_slab_box_half cells of reach), then nicr_slab_scan_apply with the
 * nuclei of the higher ranks) and nicr_slab_note_step(s, scanned), then
 * nicr_slab_end(enqueued, &completed): the status and rollback of nicr_run
 * (only the rank owning the failing cell has its message). The coloured
 * initialisation (eta_colours) needs the ranks' adjacencies OR-reduced:
 * nicr_slab_adjacency (ng x ng bytes), nicr_colour_grains, then
 * nicr_slab_set_colours on every rank. The other calls of this header
 * (fields, budget, diagnostics) see the slab's stored planes / own planes. */
int nicr_slab_create(const nicr_config* cfg, int nslabs, int index, nicr_handle** out);
int nicr_slab_info(const nicr_handle* h, int* x0, int* x1, int* x_lo, int* x_hi, int* stored, int* halo);
int nicr_slab_region(nicr_handle* h, int field, int index, int which, int width, void** ptr, long long* count);
int nicr_slab_adjacency(nicr_handle* h, unsigned char* adj);
int nicr_colour_grains(const unsigned char* adj, int ng, int k, int* colours);
int nicr_slab_set_colours(nicr_handle* h, const int* colours);
int nicr_slab_begin(nicr_handle* h, int nsteps, int schedule);
int nicr_slab_scan_due(nicr_handle* h, int s);
int nicr_slab_note_step(nicr_handle* h, int s, int scanned);
int nicr_slab_failed(nicr_handle* h, int* failed);
int nicr_slab_launch(nicr_handle* h);
void* nicr_slab_agree_word(nicr_handle* h);
int nicr_slab_commit(nicr_handle* h);
int nicr_slab_end(nicr_handle* h, int enqueued, int* completed);
int nicr_slab_scan_candidates(nicr_handle* h);
int nicr_slab_scan_resolve(nicr_handle* h, const int* pre, int npre, int* out, int cap, int* nout, int* nuclei);
int nicr_slab_scan_apply(nicr_handle* h, const int* list, int n);
int nicr_slab_box_half(const nicr_handle* h);

/* Learned surrogate building blocks (no counterpart in the reference): 3x3x3
 * convolutions, stride 1, zero padding 1, on the BF16 tensor cores with FP32
 * accumulation, on device pointers and the caller's CUDA stream. x: NDHWC
 * BF16 (n, d, h, w, cin); w: BF16 [cout][27][cin], tap = (dz+1)*9 +
 * (dy+1)*3 + (dx+1); y, dw: FP32. n*d*h*w a multiple of 64; cin and cout
 * multiples of 16. nicr_conv3d_fwd: y[v][co] = sum x[v+off(tap)][ci]
 * w[co][tap][ci]. nicr_conv3d_wgrad: dw[co][tap][ci] = sum_v dy[v][co]
 * x[v+off(tap)][ci] (dy: BF16 NDHWC with cout channels). The data gradient
 * is nicr_conv3d_fwd of dy with w'[ci][tap][co] = w[co][26-tap][ci].
 * nicr_conv3d_fwd runs on tcgen05.mma (accumulator in TMEM) with TMA-staged
 * operands (nicr_conv3d_fwd_tma, which returns NICR_ERR_INVALID_ARG when the
 * driver refuses its tensor maps) and otherwise with cp.async-gathered ones
 * (nicr_conv3d_fwd_gather); nicr_conv3d_fwd_mma_sync is the same
 * convolution on the warp-level MMA instructions. nicr_conv3d_wgrad runs on
 * tcgen05.mma with TMA-staged operands (nicr_conv3d_wgrad_tma: Cout 16, 32,
 * 64 or a multiple of 128, else NICR_ERR_INVALID_ARG) and otherwise on the
 * warp-level instructions (nicr_conv3d_wgrad_mma_sync). nicr_conv3d_error copies
 * and clears the flag the tcgen05 kernels set when one of their bounded
 * waits gives up (synchronous). */
int nicr_conv3d_fwd(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                    void* stream);
int nicr_conv3d_fwd_tma(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                        void* stream);
/* The tcgen05 forward with its epilogue fused: y = act(conv(x, w) + bias),
 * bias FP32 [cout] or NULL, act bit 1 = ReLU, bit 2 = store BF16 (else
 * FP32). NICR_ERR_INVALID_ARG where nicr_conv3d_fwd_tma would return it. */
int nicr_conv3d_fwd_act(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                        int cin, int cout, void* stream);
/* The same from a staged halo block (Cout <= 64 and rows of at least 128
 * voxels, else NICR_ERR_INVALID_ARG); nicr_conv3d_fwd_act and
 * nicr_conv3d_fwd use it for Cout <= 32 with Cin x Cout <= 768, where it is
 * the faster form. */
int nicr_conv3d_fwd_halo(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h, int w_,
                         int cin, int cout, void* stream);
/* The halo-block forward marching along y (a CTA keeps its input lines and
 * weights on chip between output lines): Cin <= 48, Cout <= 32 and rows of
 * at least 128 voxels, else NICR_ERR_INVALID_ARG; nicr_conv3d_fwd_act and
 * nicr_conv3d_fwd use it for Cin 16, where it is the fastest form. */
int nicr_conv3d_fwd_march(const void* x, const void* w, const float* bias, int act, void* y, int n, int d, int h,
                          int w_, int cin, int cout, void* stream);
int nicr_conv3d_fwd_gather(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                           void* stream);
int nicr_conv3d_fwd_mma_sync(const void* x, const void* w, float* y, int n, int d, int h, int w_, int cin, int cout,
                             void* stream);
int nicr_conv3d_wgrad(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                      void* stream);
int nicr_conv3d_wgrad_tma(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                          void* stream);
int nicr_conv3d_wgrad_mma_sync(const void* x, const void* dy, float* dw, int n, int d, int h, int w_, int cin, int cout,
                               void* stream);
int nicr_conv3d_error(int* flag);

/* The solver program: the reference's run()/main() for dim 2 or 3
 * (2D:1161-1246, 3S:1309-1395), argv as the reference's executable takes it.
 * Returns the process exit code. */
int nicr_main(int dim, int argc, const char* const* argv);

/* Stream the handle enqueues on (a cudaStream_t), for callers that overlap. */
void* nicr_stream(nicr_handle* h);

/* Measurement hooks (no counterpart in the reference, which has no GPU). When
 * enabled, CUDA events bracket every kernel launch on the handle's stream;
 * nicr_profile_read returns the accumulated device time and launch count of
 * one kernel (0 step_main, 1 eta_update, 2 step_finalize, 3 eta_mask,
 * 4 ksp_scan, 5 refresh, 6 diagnostics, 7 step_eta: the step kernel and the
 * eta update in one launch, reciprocal form; 8 step_fused: the one-pass step
 * of 3D grids with evolving eta). nicr_kernel_launches counts every
 * kernel the handle has launched since creation. */
int nicr_profile(nicr_handle* h, int enable);
int nicr_profile_read(nicr_handle* h, int kernel, double* total_ms, long long* launches);
const char* nicr_profile_kernel_name(int kernel);
long long nicr_kernel_launches(const nicr_handle* h);

/* Device self-check of the correctly rounded division by a run constant that
 * the FP64 kernels use in place of IEEE a/b: n pseudo-random numerators
 * (seeded) divided by b both ways on the current device. Returns the number
 * of results that differ (0 expected) or -1 on a CUDA error; *tested receives
 * the number of finite numerators checked. No counterpart in the reference. */
long long nicr_check_division(double b, long long n, unsigned long long seed, long long* tested);

#ifdef __cplusplus
}
#endif
#endif /* NICR_H */
