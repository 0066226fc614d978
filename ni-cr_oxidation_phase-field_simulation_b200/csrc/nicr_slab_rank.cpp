// Slab form with one process per GPU: the C-ABI of one slab of a domain split
// along X over `nslabs` ranks (the partition, halo width, initialisation and
// kernels of the one-process group, nicr_slabs.cpp). The caller owns the
// communication (nicr/slab_ranks.py: torch.distributed over NCCL):
//   per step   nicr_slab_launch    step kernels + this step's agreement word
//              (MIN collective over the ranks' agreement words)
//              nicr_slab_commit    commit with the reduced word, flip parity
//              (halo exchange: nicr_slab_region gives the device planes each
//               rank sends to / receives from its neighbours)
//   Ksp scan   nicr_slab_scan_candidates, then nicr_slab_scan_resolve rank
//              after rank in X order (the nuclei of lower ranks in `pre`),
//              then nicr_slab_scan_apply with the nuclei of higher ranks
//   schedule   nicr_slab_begin / nicr_slab_scan_due / nicr_slab_note_step /
//              nicr_slab_end: run()'s Ksp schedule and the commit or
//              rollback of a batch of steps, as nicr_run does.
// Every call is stream-ordered on the handle's stream (nicr_stream) except
// where it returns host data.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_slabs.h"

namespace nicr {

// Device planes of field/index in the current state: which = 0 the first
// `width` own planes (sent to the slab below), 1 the last own planes (sent
// above), 2 the halo planes below (received from below), 3 the halo planes
// above. Returns the device pointer and the number of doubles (width planes).
class SlabRank {
public:
    static double* region(Model& m, int field, int index, int which, int width, long long* count) {
        if (!m.is_slab) throw Error(NICR_ERR_STATE, "not a slab handle");
        if (width < 1 || which < 0 || which > 3) throw Error(NICR_ERR_INVALID_ARG, "bad region");
        const int below = m.sp.x_lo, above = m.g.nx - m.sp.x_hi, own = m.sp.x_hi - m.sp.x_lo;
        int first = 0;
        switch (which) {
            case 0: first = m.sp.x_lo; if (width > own) throw Error(NICR_ERR_INVALID_ARG, "region wider than the slab"); break;
            case 1: first = m.sp.x_hi - width; if (width > own) throw Error(NICR_ERR_INVALID_ARG, "region wider than the slab"); break;
            case 2: first = m.sp.x_lo - width; if (width > below) throw Error(NICR_ERR_INVALID_ARG, "no halo that deep below"); break;
            default: first = m.sp.x_hi; if (width > above) throw Error(NICR_ERR_INVALID_ARG, "no halo that deep above"); break;
        }
        double* base = nullptr;
        switch (field) {
            case NICR_FIELD_O: base = m.o_[m.cur]; break;
            case NICR_FIELD_CR: base = m.cr_[m.cur]; break;
            case NICR_FIELD_PHI: base = m.p_[m.cur]; break;
            case NICR_FIELD_GB: base = m.gb_[m.gcur]; break;
            case NICR_FIELD_ETA:
                if (index < 0 || index >= m.neta) throw Error(NICR_ERR_INVALID_ARG, "eta index out of range");
                base = m.eta_[m.ecur] + (size_t)index * m.g.nstore;
                break;
            default: throw Error(NICR_ERR_INVALID_ARG, "only O, CR, PHI, GB and ETA planes are exchanged");
        }
        if (count) *count = (long long)width * m.g.plane;
        return base + (size_t)first * m.g.plane;
    }
    static void set_colours(Model& m, const int* colours) {
        const int ng = (int)(m.seeds.size() / 3);
        m.seed_colour.assign(colours, colours + ng);
        m.init_eta_coloured();
        m.eta_mask_now();
    }
    static const std::vector<unsigned char>& adjacency(const Model& m) { return m.adjacency; }
    static int resolve(Model& m, const KspNucleus* pre, int npre, KspNucleus* out, int cap, int* nout) {
        KspNucleus *d_pre = nullptr, *d_out = nullptr;
        check_cuda(cudaMalloc(&d_pre, sizeof(KspNucleus) * (size_t)std::max(1, npre)), "cudaMalloc");
        check_cuda(cudaMalloc(&d_out, sizeof(KspNucleus) * (size_t)std::max(1, cap)), "cudaMalloc");
        if (npre) check_cuda(cudaMemcpyAsync(d_pre, pre, sizeof(KspNucleus) * (size_t)npre, cudaMemcpyHostToDevice, m.stream), "H2D");
        launch_ksp_resolve_slab(m.kd, d_pre, npre, d_out, cap, m.o_[m.cur], m.cr_[m.cur], m.p_[m.cur], m.eta_[m.ecur],
                                m.kw, m.bud, m.kres, m.st, m.stream);
        m.launches += 1;
        KspResult r;
        check_cuda(cudaMemcpyAsync(&r, m.kres, sizeof r, cudaMemcpyDeviceToHost, m.stream), "D2H");
        m.sync();
        const int n = std::min(r.listed, cap);
        if (n) check_cuda(cudaMemcpy(out, d_out, sizeof(KspNucleus) * (size_t)n, cudaMemcpyDeviceToHost), "D2H");
        cudaFree(d_pre);
        cudaFree(d_out);
        if (r.listed > cap) throw Error(NICR_ERR_STATE, "more nuclei in one Ksp scan of a slab than the list holds");
        *nout = r.listed;
        return r.nuclei;
    }
    static void apply(Model& m, const KspNucleus* list, int n) {
        if (n <= 0) return;
        KspNucleus* d = nullptr;
        check_cuda(cudaMalloc(&d, sizeof(KspNucleus) * (size_t)n), "cudaMalloc");
        check_cuda(cudaMemcpyAsync(d, list, sizeof(KspNucleus) * (size_t)n, cudaMemcpyHostToDevice, m.stream), "H2D");
        launch_ksp_apply(m.kd, d, n, m.o_[m.cur], m.cr_[m.cur], m.p_[m.cur], m.eta_[m.ecur], m.kw, m.bud, m.kres, m.st,
                         m.stream);
        m.launches += 1;
        m.sync();
        cudaFree(d);
    }
    static void candidates(Model& m) {
        m.kd.neta = m.neta;
        launch_ksp_candidates(m.kd, m.o_[m.cur], m.cr_[m.cur], m.p_[m.cur], m.kw, m.st, m.stream);
        m.launches += 3;
    }
    static bool failed(Model& m) {
        check_cuda(cudaMemcpyAsync(m.h_st, m.st, sizeof(Status), cudaMemcpyDeviceToHost, m.stream), "D2H");
        m.sync();
        return m.h_st->failed != 0;
    }
    static void scan_done(Model& m) {
        if (m.has_eta) m.eta_dirty = true;
        check_cuda(cudaGetLastError(), "ksp");
    }
    // ceil(r) + ceil(r + gap): how far from a nucleus its stamp and marks reach
    static int box_half(const Model& m) { return m.kd.box_half; }
};

}  // namespace nicr

namespace {

template <class F>
int rank_guarded(nicr_handle* h, F&& f) {
    if (!h || !h->m) return NICR_ERR_INVALID_ARG;
    try {
        nicr::check_cuda(cudaSetDevice(h->m->c.device), "cudaSetDevice");
        return f(*h->m);
    } catch (const nicr::Error& e) {
        h->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        h->err = e.what();
        return NICR_ERR_CUDA;
    }
}

}  // namespace

extern "C" {

int nicr_slab_create(const nicr_config* cfg, int nslabs, int index, nicr_handle** out) {
    if (!out || !cfg) return NICR_ERR_INVALID_ARG;
    *out = nullptr;
    auto* h = new nicr_handle;
    try {
        const nicr::SlabSpec q = nicr::slab_partition(*cfg, nslabs, index);
        h->m = new nicr::Model(*cfg, &q);
        *out = h;
        return NICR_OK;
    } catch (const nicr::Error& e) {
        nicr::set_create_error(e.what());
        delete h;
        return e.code;
    } catch (const std::exception& e) {
        nicr::set_create_error(e.what());
        delete h;
        return NICR_ERR_CUDA;
    }
}

int nicr_slab_info(const nicr_handle* h, int* x0, int* x1, int* x_lo, int* x_hi, int* stored, int* halo) {
    if (!h || !h->m || !h->m->is_slab) return NICR_ERR_INVALID_ARG;
    const nicr::Model& m = *h->m;
    const nicr::StepParams sp = m.params();
    if (x0) *x0 = m.x_off + sp.x_lo;
    if (x1) *x1 = m.x_off + sp.x_hi;
    if (x_lo) *x_lo = sp.x_lo;
    if (x_hi) *x_hi = sp.x_hi;
    if (stored) *stored = m.g.nx;
    if (halo) *halo = std::max(sp.x_lo, m.g.nx - sp.x_hi);
    return NICR_OK;
}

int nicr_slab_region(nicr_handle* h, int field, int index, int which, int width, void** ptr, long long* count) {
    if (!ptr) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        *ptr = nicr::SlabRank::region(m, field, index, which, width, count);
        return NICR_OK;
    });
}

int nicr_slab_adjacency(nicr_handle* h, unsigned char* adj) {
    if (!adj) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        const auto& a = nicr::SlabRank::adjacency(m);
        if (a.empty()) throw nicr::Error(NICR_ERR_STATE, "no grain adjacency (eta_colours is 0)");
        std::memcpy(adj, a.data(), a.size());
        return NICR_OK;
    });
}

int nicr_colour_grains(const unsigned char* adj, int ng, int k, int* colours) {
    if (!adj || !colours || ng < 1 || k < 1) return NICR_ERR_INVALID_ARG;
    const std::vector<unsigned char> a(adj, adj + (size_t)ng * ng);
    const std::vector<int> c = nicr::colour_grains(a, ng, k);
    std::memcpy(colours, c.data(), c.size() * sizeof(int));
    return NICR_OK;
}

int nicr_slab_set_colours(nicr_handle* h, const int* colours) {
    if (!colours) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        nicr::SlabRank::set_colours(m, colours);
        return NICR_OK;
    });
}

int nicr_slab_begin(nicr_handle* h, int nsteps, int schedule) {
    return rank_guarded(h, [&](nicr::Model& m) {
        m.run_begin(m.rank_plan, nsteps, schedule != 0);
        return NICR_OK;
    });
}

int nicr_slab_scan_due(nicr_handle* h, int s) {
    if (!h || !h->m) return 0;
    return h->m->ksp_due(h->m->rank_plan, s) ? 1 : 0;
}

int nicr_slab_note_step(nicr_handle* h, int s, int scanned) {
    return rank_guarded(h, [&](nicr::Model& m) {
        nicr::Model::RunPlan& r = m.rank_plan;
        if (!r.schedule) return NICR_OK;
        if (s < 0 || s >= r.nsteps) throw nicr::Error(NICR_ERR_INVALID_ARG, "step outside the batch");
        if (scanned) r.next += m.c.nucleation_period;
        r.sched[(size_t)s] = r.next;
        return NICR_OK;
    });
}

int nicr_slab_failed(nicr_handle* h, int* failed) {
    if (!failed) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        *failed = nicr::SlabRank::failed(m) ? 1 : 0;
        return NICR_OK;
    });
}

int nicr_slab_launch(nicr_handle* h) {
    return rank_guarded(h, [&](nicr::Model& m) {
        if (!m.is_slab) throw nicr::Error(NICR_ERR_STATE, "not a slab handle");
        m.rank_launch();
        return NICR_OK;
    });
}

void* nicr_slab_agree_word(nicr_handle* h) {
    if (!h || !h->m) return nullptr;
    try {
        nicr::check_cuda(cudaSetDevice(h->m->c.device), "cudaSetDevice");
        return static_cast<void*>(h->m->d_agree());
    } catch (...) {
        return nullptr;
    }
}

int nicr_slab_commit(nicr_handle* h) {
    return rank_guarded(h, [&](nicr::Model& m) {
        m.rank_commit();
        return NICR_OK;
    });
}

int nicr_slab_end(nicr_handle* h, int enqueued, int* completed) {
    return rank_guarded(h, [&](nicr::Model& m) {
        nicr::Model::RunPlan& r = m.rank_plan;
        r.nsteps = std::min(r.nsteps, std::max(0, enqueued));
        const int rc = m.run_end(r, completed);
        if (rc != NICR_OK) throw nicr::Error(rc, m.last_error);
        return NICR_OK;
    });
}

int nicr_slab_scan_candidates(nicr_handle* h) {
    return rank_guarded(h, [&](nicr::Model& m) {
        nicr::SlabRank::candidates(m);
        return NICR_OK;
    });
}

int nicr_slab_scan_resolve(nicr_handle* h, const int* pre, int npre, int* out, int cap, int* nout, int* nuclei) {
    if ((npre > 0 && !pre) || !out || !nout || cap < 0) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        const int k = nicr::SlabRank::resolve(m, reinterpret_cast<const nicr::KspNucleus*>(pre), npre,
                                              reinterpret_cast<nicr::KspNucleus*>(out), cap, nout);
        if (nuclei) *nuclei = k;
        return NICR_OK;
    });
}

int nicr_slab_scan_apply(nicr_handle* h, const int* list, int n) {
    if (n > 0 && !list) return NICR_ERR_INVALID_ARG;
    return rank_guarded(h, [&](nicr::Model& m) {
        nicr::SlabRank::apply(m, reinterpret_cast<const nicr::KspNucleus*>(list), n);
        nicr::SlabRank::scan_done(m);
        return NICR_OK;
    });
}

int nicr_slab_box_half(const nicr_handle* h) { return h && h->m ? nicr::SlabRank::box_half(*h->m) : 0; }

}  // extern "C"
