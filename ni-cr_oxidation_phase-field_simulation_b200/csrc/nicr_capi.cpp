// extern "C" entry points of include/nicr.h. Exceptions never cross this
// boundary: every call maps failures to a status code and keeps the message
// for nicr_last_error.
#include <cstring>
#include <new>
#include <string>

#include "../../include/nicr.h"
#include "nicr_model.h"


namespace {
thread_local std::string g_create_error;
}  // namespace

// the message nicr_last_error(NULL) returns after a failed creation
void nicr::set_create_error(const std::string& e) { g_create_error = e; }

namespace {

template <class Fn>
int guarded(nicr_handle* h, Fn fn) {
    if (!h || !h->m) return NICR_ERR_INVALID_ARG;
    try {
        const int rc = fn(*h->m);
        if (rc != NICR_OK) h->err = h->m->last_error;
        return rc;
    } catch (const nicr::Error& e) {
        h->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return NICR_ERR_STATE;
    } catch (const std::exception& e) {
        h->err = e.what();
        return NICR_ERR_STATE;
    }
}
}  // namespace

extern "C" {

int nicr_create(const nicr_config* cfg, nicr_handle** out) {
    if (!cfg || !out) return NICR_ERR_INVALID_ARG;
    *out = nullptr;
    try {
        auto* h = new nicr_handle;
        try {
            h->m = new nicr::Model(*cfg);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return NICR_OK;
    } catch (const nicr::Error& e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return NICR_ERR_STATE;
    }
}

void nicr_destroy(nicr_handle* h) {
    if (!h || h->borrowed) return;
    delete h->m;
    delete h;
}

const char* nicr_last_error(const nicr_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int nicr_get_info(const nicr_handle* hc, nicr_info* info) {
    auto* h = const_cast<nicr_handle*>(hc);
    return guarded(h, [&](nicr::Model& m) {
        if (!info) return (int)NICR_ERR_INVALID_ARG;
        info->dim = m.dim;
        info->nx = m.c.nx; info->ny = m.c.ny; info->nz = m.dim == 3 ? m.c.nz : 1;
        info->n_seeds = (int)(m.seeds.size() / m.dim);
        info->n_eta = m.neta;
        info->center_seed_cells = m.center_seed_cells;
        info->grain_map_retained = m.grain_retained ? 1 : 0;
        info->n_cells = m.g.ncells;
        info->steps_done = m.steps_done;
        info->device_bytes = m.device_bytes();
        return (int)NICR_OK;
    });
}

int nicr_get_seeds(const nicr_handle* hc, double* xyz, long long* volumes) {
    auto* h = const_cast<nicr_handle*>(hc);
    return guarded(h, [&](nicr::Model& m) {
        if (xyz) std::memcpy(xyz, m.seeds.data(), m.seeds.size() * sizeof(double));
        if (volumes) std::memcpy(volumes, m.volumes.data(), m.volumes.size() * sizeof(long long));
        return (int)NICR_OK;
    });
}

int nicr_set_field(nicr_handle* h, int field, int index, const double* host) {
    return guarded(h, [&](nicr::Model& m) {
        if (!host) return (int)NICR_ERR_INVALID_ARG;
        m.set_field(field, index, host);   // mu/M and a stale eta mask are recomputed when next needed
        return (int)NICR_OK;
    });
}

int nicr_get_field(nicr_handle* h, int field, int index, double* host) {
    return guarded(h, [&](nicr::Model& m) {
        if (!host) return (int)NICR_ERR_INVALID_ARG;
        m.get_field(field, index, host);
        return (int)NICR_OK;
    });
}

int nicr_save_state(nicr_handle* h, const char* path) {
    return guarded(h, [&](nicr::Model& m) {
        if (!path) return (int)NICR_ERR_INVALID_ARG;
        m.save_state(path);
        return (int)NICR_OK;
    });
}

int nicr_load_state(nicr_handle* h, const char* path) {
    return guarded(h, [&](nicr::Model& m) {
        if (!path) return (int)NICR_ERR_INVALID_ARG;
        m.load_state(path);
        return (int)NICR_OK;
    });
}

int nicr_tune(nicr_handle* h, int reps, int* xchunk, int* minb) {
    return guarded(h, [&](nicr::Model& m) {
        m.tune(reps, xchunk, minb);
        return (int)NICR_OK;
    });
}

int nicr_refresh(nicr_handle* h) {
    return guarded(h, [&](nicr::Model& m) { m.refresh(); m.sync(); return (int)NICR_OK; });
}
int nicr_field_device(nicr_handle* h, int field, int index, int writable, void** ptr, long long* pitch) {
    return guarded(h, [&](nicr::Model& m) {
        if (!ptr || !pitch) return (int)NICR_ERR_INVALID_ARG;
        if (m.is_slab) throw nicr::Error(NICR_ERR_STATE, "device views are of whole-domain handles (slabs: nicr_slab_region)");
        if (writable) {
            *ptr = m.state_ptr(field, index);
            m.invalidate_eta_cache();   // as after nicr_set_field
        } else {
            *ptr = const_cast<double*>(m.field_ptr(field, index));   // may materialise the eta mask
        }
        m.sync();
        *pitch = m.g.pb;
        return (int)NICR_OK;
    });
}

int nicr_invalidate_eta_cache(nicr_handle* h) {
    return guarded(h, [&](nicr::Model& m) { m.invalidate_eta_cache(); return (int)NICR_OK; });
}
int nicr_reset_inventory(nicr_handle* h) {
    return guarded(h, [&](nicr::Model& m) { m.reset_inventory(); return (int)NICR_OK; });
}
int nicr_step(nicr_handle* h, int nsteps, int* completed) {
    return guarded(h, [&](nicr::Model& m) { return m.step(nsteps, completed); });
}
int nicr_run(nicr_handle* h, int nsteps, int* completed) {
    return guarded(h, [&](nicr::Model& m) { return m.run(nsteps, completed); });
}
int nicr_nucleate(nicr_handle* h, int* nuclei) {
    return guarded(h, [&](nicr::Model& m) { return m.nucleate(nuclei); });
}
int nicr_stamp(nicr_handle* h, int x, int y, int z, int* cells) {
    return guarded(h, [&](nicr::Model& m) { return m.stamp(x, y, z, cells); });
}
int nicr_get_budget(const nicr_handle* hc, nicr_budget* b) {
    auto* h = const_cast<nicr_handle*>(hc);
    return guarded(h, [&](nicr::Model& m) {
        if (!b) return (int)NICR_ERR_INVALID_ARG;
        m.budget(b);
        return (int)NICR_OK;
    });
}
int nicr_get_diagnostics(nicr_handle* h, nicr_diagnostics* d) {
    return guarded(h, [&](nicr::Model& m) {
        if (!d) return (int)NICR_ERR_INVALID_ARG;
        m.diagnostics(d);
        return (int)NICR_OK;
    });
}
int nicr_get_grain_stats(nicr_handle* h, nicr_grain_stats* s, long long* cells, double* amount) {
    return guarded(h, [&](nicr::Model& m) {
        if (!s) return (int)NICR_ERR_INVALID_ARG;
        m.grain_stats(s, cells, amount);
        return (int)NICR_OK;
    });
}

int nicr_profile(nicr_handle* h, int enable) {
    return guarded(h, [&](nicr::Model& m) { m.profile_enable(enable != 0); return (int)NICR_OK; });
}

int nicr_profile_read(nicr_handle* h, int kernel, double* total_ms, long long* launches) {
    return guarded(h, [&](nicr::Model& m) {
        if (kernel < 0 || kernel >= nicr::Model::K_COUNT) return (int)NICR_ERR_INVALID_ARG;
        m.profile_collect();
        if (total_ms) *total_ms = m.prof_ms[kernel];
        if (launches) *launches = m.prof_n[kernel];
        return (int)NICR_OK;
    });
}

const char* nicr_profile_kernel_name(int kernel) { return nicr::Model::kernel_name(kernel); }

long long nicr_kernel_launches(const nicr_handle* h) { return (h && h->m) ? h->m->launches : -1; }

long long nicr_check_division(double b, long long n, unsigned long long seed, long long* tested) {
    return nicr::check_division(b, n, seed, tested);
}

void* nicr_stream(nicr_handle* h) { return (h && h->m) ? (void*)h->m->stream : nullptr; }

}  // extern "C"
