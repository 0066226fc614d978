// Batched multi-domain form: many independent domains of one device advanced
// together. Each domain is an ordinary Model (its own buffers, initialisation,
// Ksp schedule, budgets and failure handling, all identical to a single
// handle); what the batch changes is the launch structure of a step: one
// k_step_batch launch per group of up to kBatchMax domains instead of one
// step launch per domain, and one finalize launch for all domains, all on the
// batch's stream. Small domains (32^3..96^3) would otherwise leave the GPU
// launch-bound and mostly idle.
#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_model.h"

struct nicr_batch {
    std::vector<nicr_handle*> doms;
    cudaStream_t stream = nullptr;
    int device = 0;
    std::string err;
    long long launches = 0;   // batch-level launches (grouped step + finalize)

    ~nicr_batch() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& q : graphs)
            if (q.exec) cudaGraphExecDestroy(q.exec);
        for (nicr_handle* h : doms) {
            delete h->m;
            delete h;
        }
        if (stream) cudaStreamDestroy(stream);
    }

    // Step pairs of the whole batch captured as CUDA graphs, one per parity
    // state of all domains (they toggle together; a domain that was rolled
    // back after a failed trial may differ), replayed when no domain scans
    // for Ksp in either step. Each graph holds the grouped step launches, the
    // domains' eta updates and the batched commit of two steps.
    struct PairGraph {
        std::vector<int> key;
        cudaGraphExec_t exec = nullptr;
        long long batch_kernels = 0;
        std::vector<long long> domain_kernels;
    };
    std::vector<PairGraph> graphs;

    void enqueue_step(std::vector<nicr::BatchDomain>& descs, std::vector<nicr::FinalizeDomain>& fins) {
        const int n = (int)doms.size();
        for (int i = 0; i < n; ++i) {
            nicr::Model& m = *doms[i]->m;
            m.prepare_step();
            descs[i] = m.step_desc();
        }
        launches += nicr::launch_step_batch(descs.data(), n, stream);
        for (int i = 0; i < n; ++i) {
            nicr::Model& m = *doms[i]->m;
            m.complete_step(descs[i].nblocks, false);
            fins[i] = m.finalize_desc(descs[i].nblocks);
        }
        nicr::launch_finalize_batch(fins.data(), n, stream);
        launches += (n + nicr::kFinalizeMax - 1) / nicr::kFinalizeMax;
    }

    void launch_pair(std::vector<nicr::BatchDomain>& descs, std::vector<nicr::FinalizeDomain>& fins) {
        const int n = (int)doms.size();
        std::vector<int> key((size_t)n);
        for (int i = 0; i < n; ++i) {
            doms[i]->m->prepare_step();   // stale eta masks are rebuilt outside the graph
            key[i] = doms[i]->m->parity_key();
        }
        PairGraph* pg = nullptr;
        for (auto& q : graphs)
            if (q.key == key) pg = &q;
        if (!pg) {
            if (graphs.size() >= 4) {   // parities this varied: drop the oldest capture
                cudaGraphExecDestroy(graphs.front().exec);
                graphs.erase(graphs.begin());
            }
            for (auto* h : doms) nicr::step_kernels_prepare(h->m->params());
            PairGraph q;
            q.key = key;
            const long long b0 = launches;
            std::vector<long long> d0((size_t)n);
            for (int i = 0; i < n; ++i) d0[i] = doms[i]->m->launches;
            cudaGraph_t graph = nullptr;
            nicr::check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            enqueue_step(descs, fins);
            enqueue_step(descs, fins);
            nicr::check_cuda(cudaStreamEndCapture(stream, &graph), "cudaStreamEndCapture");
            const cudaError_t e = cudaGraphInstantiate(&q.exec, graph, 0);
            cudaGraphDestroy(graph);
            nicr::check_cuda(e, "cudaGraphInstantiate");
            // nothing ran while capturing: each replay counts the kernels
            q.batch_kernels = launches - b0;
            launches = b0;
            q.domain_kernels.resize((size_t)n);
            for (int i = 0; i < n; ++i) {
                q.domain_kernels[i] = doms[i]->m->launches - d0[i];
                doms[i]->m->launches = d0[i];
            }
            graphs.push_back(std::move(q));
            pg = &graphs.back();
        }
        nicr::check_cuda(cudaGraphLaunch(pg->exec, stream), "cudaGraphLaunch");
        launches += pg->batch_kernels;
        for (int i = 0; i < n; ++i) doms[i]->m->launches += pg->domain_kernels[i];
    }

    // The batch's common X chunk by measurement: `reps` timed passes of the
    // grouped step launches and the domains' eta updates per candidate, on
    // the current states, into the trial buffers only.
    int tune(int reps, int* chunk_out) {
        const int n = (int)doms.size();
        reps = std::max(1, reps);
        int nxmax = 1;
        for (auto* h : doms) {
            h->m->prepare_step();
            nxmax = std::max(nxmax, h->m->g.nx);
        }
        std::vector<nicr::BatchDomain> descs((size_t)n);
        cudaEvent_t e0, e1;
        nicr::check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        nicr::check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        auto pass = [&] {
            for (int i = 0; i < n; ++i) descs[i] = doms[i]->m->step_desc();
            nicr::launch_step_batch(descs.data(), n, stream);
            for (auto* h : doms)
                if (h->m->advance_eta) h->m->launch_trial_eta();   // the step kernel ran batched above
        };
        int best = doms[0]->m->params().xchunk;
        float best_ms = -1.f;
        for (int c : nicr::xchunk_candidates(nxmax)) {
            for (auto* h : doms) h->m->set_xchunk(c);
            pass();
            nicr::check_cuda(cudaEventRecord(e0, stream), "cudaEventRecord");
            for (int r = 0; r < reps; ++r) pass();
            nicr::check_cuda(cudaEventRecord(e1, stream), "cudaEventRecord");
            nicr::check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            nicr::check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            if (best_ms < 0.f || ms < best_ms) { best_ms = ms; best = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        nicr::check_cuda(cudaGetLastError(), "tune");
        for (auto* h : doms) h->m->set_xchunk(best);
        for (auto& q : graphs)
            if (q.exec) cudaGraphExecDestroy(q.exec);
        graphs.clear();
        if (chunk_out) *chunk_out = best;
        return NICR_OK;
    }

    // Advances every domain nsteps steps (run() schedule when `schedule`).
    int advance(int nsteps, int* completed, bool schedule) {
        const int n = (int)doms.size();
        if (completed)
            for (int i = 0; i < n; ++i) completed[i] = 0;
        if (nsteps <= 0) return NICR_OK;
        std::vector<nicr::Model::RunPlan> plans((size_t)n);
        std::vector<nicr::BatchDomain> descs((size_t)n);
        std::vector<nicr::FinalizeDomain> fins((size_t)n);
        for (int i = 0; i < n; ++i) doms[i]->m->run_begin(plans[i], nsteps, schedule);
        const bool use_graphs = doms[0]->m->graphs_enabled();
        for (int s = 0; s < nsteps;) {
            for (int i = 0; i < n; ++i) doms[i]->m->run_pre_step(plans[i], s);
            bool pair = use_graphs && s + 1 < nsteps;
            for (int i = 0; pair && i < n; ++i) pair = !doms[i]->m->ksp_due(plans[i], s + 1);
            if (pair) {
                launch_pair(descs, fins);
                for (int i = 0; i < n; ++i) doms[i]->m->run_pre_step(plans[i], s + 1);   // schedule entry only
                s += 2;
            } else {
                enqueue_step(descs, fins);
                ++s;
            }
        }
        int rc = NICR_OK;
        err.clear();
        for (int i = 0; i < n; ++i) {
            nicr::Model& m = *doms[i]->m;
            const int r = m.run_end(plans[i], completed ? completed + i : nullptr);
            if (r != NICR_OK) {
                doms[i]->err = m.last_error;
                if (rc == NICR_OK) {
                    rc = r;
                    err = "domain " + std::to_string(i) + ": " + m.last_error;
                }
            }
        }
        return rc;
    }
};

namespace {
thread_local std::string g_batch_error;

template <class Fn>
int batch_guarded(nicr_batch* b, Fn fn) {
    if (!b) return NICR_ERR_INVALID_ARG;
    try {
        return fn(*b);
    } catch (const nicr::Error& e) {
        b->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        b->err = "host allocation failed";
        return NICR_ERR_STATE;
    } catch (const std::exception& e) {
        b->err = e.what();
        return NICR_ERR_STATE;
    }
}
}  // namespace

extern "C" {

int nicr_batch_create(const nicr_config* cfgs, int n, nicr_batch** out) {
    if (!out) return NICR_ERR_INVALID_ARG;
    *out = nullptr;
    if (!cfgs || n <= 0) {
        g_batch_error = "a batch needs at least one configuration";
        return NICR_ERR_INVALID_ARG;
    }
    for (int i = 1; i < n; ++i)
        if (cfgs[i].device != cfgs[0].device) {
            g_batch_error = "all domains of a batch must use the same device";
            return NICR_ERR_INVALID_ARG;
        }
    nicr_batch* b = nullptr;
    try {
        b = new nicr_batch;
        b->device = cfgs[0].device;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || b->device < 0 || b->device >= count) {
            delete b;
            g_batch_error = "no CUDA device " + std::to_string(cfgs[0].device);
            return NICR_ERR_NO_DEVICE;
        }
        nicr::check_cuda(cudaSetDevice(b->device), "cudaSetDevice");
        nicr::check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        b->doms.reserve((size_t)n);
        for (int i = 0; i < n; ++i) {
            auto* h = new nicr_handle;
            h->borrowed = true;
            try {
                h->m = new nicr::Model(cfgs[i]);
            } catch (...) {
                delete h;
                throw;
            }
            b->doms.push_back(h);
            h->m->adopt_stream(b->stream);
        }
        // the domains share the GPU: one X chunk for all, from their total CTAs
        std::vector<nicr::Grid> grids;
        for (nicr_handle* h : b->doms) grids.push_back(h->m->g);
        const int chunk = nicr::choose_xchunk_batch(grids.data(), (int)grids.size());
        for (nicr_handle* h : b->doms) h->m->set_xchunk(chunk);
        *out = b;
        return NICR_OK;
    } catch (const nicr::Error& e) {
        g_batch_error = e.what();
        delete b;
        return e.code;
    } catch (const std::exception& e) {
        g_batch_error = e.what();
        delete b;
        return NICR_ERR_STATE;
    }
}

void nicr_batch_destroy(nicr_batch* b) { delete b; }

int nicr_batch_size(const nicr_batch* b) { return b ? (int)b->doms.size() : 0; }

nicr_handle* nicr_batch_domain(nicr_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->doms.size()) return nullptr;
    return b->doms[(size_t)i];
}

int nicr_batch_step(nicr_batch* b, int nsteps, int* completed) {
    return batch_guarded(b, [&](nicr_batch& bb) { return bb.advance(nsteps, completed, false); });
}

int nicr_batch_tune(nicr_batch* b, int reps, int* xchunk) {
    return batch_guarded(b, [&](nicr_batch& bb) { return bb.tune(reps, xchunk); });
}

int nicr_batch_run(nicr_batch* b, int nsteps, int* completed) {
    return batch_guarded(b, [&](nicr_batch& bb) { return bb.advance(nsteps, completed, true); });
}

const char* nicr_batch_last_error(const nicr_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

long long nicr_batch_kernel_launches(const nicr_batch* b) {
    if (!b) return 0;
    long long n = b->launches;
    for (const nicr_handle* h : b->doms) n += h->m->launches;
    return n;
}

void* nicr_batch_stream(const nicr_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

}  // extern "C"
