// The reciprocal-division form (NICR_FP64_FAST) of the step and eta kernels.
// This unit is compiled with FMA contraction (nvcc -fmad=true): the form
// already trades bit-identity for speed (division by a run constant becomes a
// multiplication by its rounded reciprocal), and fused multiply-adds change
// its results by a few ulp per step, far inside the 1e-4 bound against the
// drop-in form (measured 4e-16 after 203 steps at 256^3), for 3-4% less time
// in both kernels on B200. The kernels are the shared templates of
// nicr_step_impl.cuh, instantiated with FAST = true.
#include "nicr_step_impl.cuh"
#include "nicr_step_fused.cuh"

namespace nicr {

void launch_step_main_fast(const StepParams& P, const double* o, const double* cr, const double* p, const double* gb,
                           const double* s2, double* on, double* crn, double* pn, StepPartial* partials, Status* st,
                           cudaStream_t stream, int* nblocks_out) {
    launch_step_form<true>(P, o, cr, p, gb, s2, on, crn, pn, partials, st, stream, nblocks_out);
}

void launch_eta_update_fast(const StepParams& P, int neta, const double* eta, const double* s2, const double* p,
                            double* eta_next, double* gb_next, double* s2_next, Status* st, cudaStream_t stream) {
    launch_eta_form<true>(P, neta, eta, s2, p, eta_next, gb_next, s2_next, st, stream);
}

bool launch_step_eta_fast(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                          const double* gb, const double* s2, double* on, double* crn, double* pn,
                          StepPartial* partials, const double* eta, double* eta_next, double* gb_next,
                          double* s2_next, unsigned* ticket, Status* st, cudaStream_t stream, int* nblocks_out) {
    return launch_step_eta_form<true>(P, neta, o, cr, p, gb, s2, on, crn, pn, partials, eta, eta_next, gb_next,
                                      s2_next, ticket, st, stream, nblocks_out);
}

bool launch_step_fused_fast(const StepParams& P, int neta, const double* o, const double* cr, const double* p,
                            const double* eta, double* on, double* crn, double* pn, double* eta_next,
                            StepPartial* partials, Status* st, cudaStream_t stream, int* nblocks_out) {
    return launch_step_fused_form<true>(P, neta, o, cr, p, eta, on, crn, pn, eta_next, partials, st, stream,
                                        nblocks_out);
}

void step_fused_prepare_fast(const StepParams& P, int neta) {
    if (fused_step_applies(P.g, neta)) step_fused_prepare<true>(neta);
}

void step_eta_prepare_fast(const StepParams& P, int neta) {
    if (P.g.dim == 3) step_eta_prepare<true>(neta);
}

void launch_batch_slim_fast(const StepBatchSlim& B, int nblocks, int dim, cudaStream_t stream) {
    if (dim == 3) launch_batch_slim<3, TA3, TB3, 2, true>(B, nblocks, stream);
    else launch_batch_slim<2, TA2, TB2, 4, true>(B, nblocks, stream);
}

void launch_batch_group_fast(StepBatch& B, int nblocks, int dim, cudaStream_t stream) {
    if (dim == 3) launch_batch_group<3, TA3, TB3, 2, true>(B, nblocks, stream);
    else launch_batch_group<2, TA2, TB2, 4, true>(B, nblocks, stream);
}

void step_kernels_prepare_fast(const StepParams& P) {
    if (P.g.dim != 3) return;   // the 2D tile fits the default 48 KB
    using T = Tile<3, TA3, TB3>;
    const void* k = step_minb_for(P) == 3 ? (const void*)k_step_main<3, TA3, TB3, 3, true>
                                     : (const void*)k_step_main<3, TA3, TB3, 2, true>;
    ensure_smem_attr(k, (int)T::SMEM_BYTES);
}

}  // namespace nicr
