// Slab form: one 3D domain split along X into slabs, the reference's own
// decomposition (mpi3d-slab/NiCr3D_grains.cpp: each MPI rank owns a range of
// X planes and trades ghost planes with its neighbours, 3S:146-191), with one
// slab per GPU in one process, or several slabs on one GPU.
//
// Each slab is an ordinary Model (nicr_model.cpp) that stores its own planes
// plus `halo` planes of each neighbour, initialised like the whole domain's
// (every initial value depends on the cell alone), so all stored copies start
// equal. One step of the group:
//   1. every slab: step kernel + eta update into its trial buffers, the
//      failing-trial key going to its error word of this step;
//   2. every slab: commit after every slab's step kernels finished (stream
//      waits on the other slabs' events). The commit reads all slabs' error
//      words of the step (peer memory for slabs on other GPUs), so all slabs
//      accept or reject alike, with the minimum key (whole-domain order);
//   3. every slab: its boundary planes of the new state are stored into the
//      neighbours' halo planes by one copy kernel (P2P stores over NVLink for
//      slabs on other GPUs); the neighbours' next step waits for it.
// No host round trip per step. Ksp scans (every nucleation period) run the
// ordered resolve slab after slab along X, which is the domain's cell order:
// each slab first applies the nuclei that slabs below it accepted in this
// scan (their stamps on its cells and their exclusion marks), then resolves
// its own candidates, and finally stamps the nuclei that slabs above it
// accepted. The stored fields are then those of a whole-domain run, bit for
// bit in the drop-in form (the reciprocal form's slab kernel instances are
// contracted to FMA apart from the whole-domain ones and may round a few
// cells differently); budgets are the sums of the slabs' double-double budgets.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_slabs.h"

namespace nicr {

namespace {
// the halo width: the step's stencil reach (2 planes of o and cr), or the
// reach of the Ksp pre-scan test, ceil(r + gap) planes of phi
int halo_for(const nicr_config& c) {
    int h = 2;
    if (c.nucleation == NICR_NUC_KSP) h = std::max(h, (int)std::ceil(c.radius_grid + c.exclusion_gap_grid));
    return h;
}
DD dd(const double* v) { return DD{v[0], v[1]}; }
void put(double* v, DD a) { v[0] = a.hi; v[1] = a.lo; }
// first-in-order extremum of two slabs' values (the lower slab wins ties, NaN loses)
double pick_min(double a, double b) {
    if (b < a) return b;
    if (a < b || a == b) return a;
    return std::isnan(a) ? b : a;
}
double pick_max(double a, double b) {
    if (a < b) return b;
    if (b < a || a == b) return a;
    return std::isnan(a) ? b : a;
}
}  // namespace

SlabSpec slab_partition(const nicr_config& c, int n, int index) {
    if (c.dim != 3) throw Error(NICR_ERR_INVALID_ARG, "the slab form is 3D only");
    if (n < 1 || n > kMaxSlabs) throw Error(NICR_ERR_INVALID_ARG, "between 1 and 16 slabs");
    if (index < 0 || index >= n) throw Error(NICR_ERR_INVALID_ARG, "slab index out of range");
    SlabSpec q;
    q.halo = halo_for(c);
    const int base = c.nx / n, rem = c.nx % n;
    if (base < q.halo)
        throw Error(NICR_ERR_INVALID_ARG, "each slab needs at least " + std::to_string(q.halo) + " planes along X");
    q.x0 = index * base + std::min(index, rem);
    q.x1 = q.x0 + base + (index < rem ? 1 : 0);
    return q;
}

SlabGroup::SlabGroup(const nicr_config& cfg, int n, const int* devices) : c(cfg) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw Error(NICR_ERR_NO_DEVICE, "no CUDA device is available");
    for (int s = 0; s < n; ++s) {
        const SlabSpec q = slab_partition(c, n, s);
        halo = q.halo;
        const int d = devices ? devices[s] : c.device;
        if (d < 0 || d >= count) throw Error(NICR_ERR_NO_DEVICE, "no CUDA device " + std::to_string(d));
        dev.push_back(d);
        x0.push_back(q.x0);
        x1.push_back(q.x1);
    }
    if (n < 1) throw Error(NICR_ERR_INVALID_ARG, "between 1 and 16 slabs");
    // every slab reads every other slab's error words, and neighbours store
    // into each other's halos: peer access between all devices in use
    for (int a : dev)
        for (int b : dev) {
            if (a == b) continue;
            int ok = 0;
            check_cuda(cudaDeviceCanAccessPeer(&ok, a, b), "cudaDeviceCanAccessPeer");
            if (!ok) throw Error(NICR_ERR_NO_DEVICE, "GPU " + std::to_string(a) + " cannot access GPU " + std::to_string(b));
            check_cuda(cudaSetDevice(a), "cudaSetDevice");
            const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            else check_cuda(e, "cudaDeviceEnablePeerAccess");
        }
    try {
        for (int s = 0; s < n; ++s) {
            nicr_config cs = c;
            cs.device = dev[(size_t)s];
            SlabSpec q;
            q.x0 = x0[(size_t)s];
            q.x1 = x1[(size_t)s];
            q.halo = halo;
            m.push_back(std::make_unique<Model>(cs, &q));
        }
        if (m[0]->has_eta && c.eta_colours > 0) {
            // every face between two planes lies in some slab's stored planes:
            // the union of the slabs' adjacencies is the domain's
            std::vector<unsigned char> adj = m[0]->adjacency;
            for (auto& q : m)
                for (size_t i = 0; i < adj.size(); ++i) adj[i] = adj[i] | q->adjacency[i];
            const std::vector<int> colours = colour_grains(adj, (int)(m[0]->seeds.size() / 3), c.eta_colours);
            for (int s = 0; s < n; ++s) {
                on(s);
                m[(size_t)s]->seed_colour = colours;
                m[(size_t)s]->init_eta_coloured();
                m[(size_t)s]->eta_mask_now();
            }
        }
        if (c.nucleation == NICR_NUC_CENTER) {
            long long cells = 0;
            for (auto& q : m) cells += q->center_seed_cells;
            if (cells == 0) throw Error(NICR_ERR_INVALID_ARG, "Center seed covers no cell centres: increase --radius-grid.");
        }
        peers.n = n;
        for (int s = 0; s < n; ++s) peers.st[s] = m[(size_t)s]->st;
        ev_done.assign((size_t)n, nullptr);
        ev_push.assign((size_t)n, nullptr);
        d_pre.assign((size_t)n, nullptr);
        d_out.assign((size_t)n, nullptr);
        for (int s = 0; s < n; ++s) {
            on(s);
            check_cuda(cudaEventCreateWithFlags(&ev_done[(size_t)s], cudaEventDisableTiming), "cudaEventCreate");
            check_cuda(cudaEventCreateWithFlags(&ev_push[(size_t)s], cudaEventDisableTiming), "cudaEventCreate");
            if (c.nucleation == NICR_NUC_KSP) {
                check_cuda(cudaMalloc(&d_pre[(size_t)s], (size_t)cap * sizeof(KspNucleus)), "cudaMalloc");
                check_cuda(cudaMalloc(&d_out[(size_t)s], (size_t)cap * sizeof(KspNucleus)), "cudaMalloc");
            }
        }
    } catch (...) {
        for (size_t s = 0; s < ev_done.size(); ++s) {
            if (ev_done[s]) cudaEventDestroy(ev_done[s]);
            if (ev_push[s]) cudaEventDestroy(ev_push[s]);
            if (d_pre[s]) cudaFree(d_pre[s]);
            if (d_out[s]) cudaFree(d_out[s]);
        }
        throw;
    }
}

SlabGroup::~SlabGroup() {
    for (size_t s = 0; s < m.size(); ++s) {
        cudaSetDevice(dev[s]);
        m[s]->sync();
        if (ev_done[s]) cudaEventDestroy(ev_done[s]);
        if (ev_push[s]) cudaEventDestroy(ev_push[s]);
        if (d_pre[s]) cudaFree(d_pre[s]);
        if (d_out[s]) cudaFree(d_out[s]);
    }
    for (size_t s = 0; s < m.size(); ++s) {
        cudaSetDevice(dev[s]);
        m[s].reset();
    }
}

long long SlabGroup::launches() const {
    long long n = copies;
    for (auto& q : m) n += q->launches;
    return n;
}

void SlabGroup::sync_all() {
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        m[(size_t)s]->sync();
    }
}

bool SlabGroup::any_failed() {
    bool f = false;
    for (int s = 0; s < (int)m.size(); ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        check_cuda(cudaMemcpyAsync(a.h_st, a.st, sizeof(Status), cudaMemcpyDeviceToHost, a.stream), "D2H");
        a.sync();
        f = f || a.h_st->failed;
    }
    return f;
}

// Stores slab s's boundary planes of the current state into its neighbours'
// halo planes: o and cr two planes deep, phi, gb and eta one (what the step
// kernels read), or phi p_width planes deep alone (before a Ksp scan).
void SlabGroup::push(int s, bool step_fields, int p_width) {
    Model& a = *m[(size_t)s];
    CopyList L{};
    const long long plane = a.g.plane;
    auto add = [&](const double* src, double* dst, int w, long long rows, long long sp, long long dp) {
        CopySeg& q = L.s[L.count++];
        q.src = src; q.dst = dst; q.n = w * plane; q.rows = rows; q.src_pitch = sp; q.dst_pitch = dp;
    };
    for (int side = 0; side < 2; ++side) {
        const int t = side == 0 ? s - 1 : s + 1;
        if (t < 0 || t >= (int)m.size()) continue;
        Model& b = *m[(size_t)t];
        // w own planes next to neighbour t -> the halo planes of t that mirror them
        auto from = [&](int w) { return (long long)(side == 0 ? a.sp.x_lo : a.sp.x_hi - w) * plane; };
        auto to = [&](int w) { return (long long)(side == 0 ? b.sp.x_hi : b.sp.x_lo - w) * plane; };
        if (step_fields) {
            add(a.o_[a.cur] + from(2), b.o_[b.cur] + to(2), 2, 1, 0, 0);
            add(a.cr_[a.cur] + from(2), b.cr_[b.cur] + to(2), 2, 1, 0, 0);
            add(a.p_[a.cur] + from(1), b.p_[b.cur] + to(1), 1, 1, 0, 0);
            if (a.advance_eta) {
                add(a.gb_[a.gcur] + from(1), b.gb_[b.gcur] + to(1), 1, 1, 0, 0);
                add(a.eta_[a.ecur] + from(1), b.eta_[b.ecur] + to(1), 1, a.neta, a.g.nstore, b.g.nstore);
            }
        } else {
            add(a.p_[a.cur] + from(p_width), b.p_[b.cur] + to(p_width), p_width, 1, 0, 0);
        }
    }
    if (L.count == 0) return;
    launch_copy_segments(L, a.st, a.stream);
    ++copies;
}

void SlabGroup::one_step() {
    const int n = (int)m.size();
    std::vector<int> nb((size_t)n, 0);
    for (int s = 0; s < n; ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        if (pushed) {
            if (s > 0) check_cuda(cudaStreamWaitEvent(a.stream, ev_push[(size_t)s - 1], 0), "cudaStreamWaitEvent");
            if (s + 1 < n) check_cuda(cudaStreamWaitEvent(a.stream, ev_push[(size_t)s + 1], 0), "cudaStreamWaitEvent");
        }
        nb[(size_t)s] = a.slab_launch();
        check_cuda(cudaEventRecord(ev_done[(size_t)s], a.stream), "cudaEventRecord");
    }
    for (int s = 0; s < n; ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        for (int j = 0; j < n; ++j)
            if (j != s) check_cuda(cudaStreamWaitEvent(a.stream, ev_done[(size_t)j], 0), "cudaStreamWaitEvent");
        a.slab_commit(nb[(size_t)s], peers);
    }
    // after every commit: the buffer parities the pushes address are the new
    // state's on both sides
    for (int s = 0; s < n; ++s) {
        on(s);
        push(s, true, 0);
        check_cuda(cudaEventRecord(ev_push[(size_t)s], m[(size_t)s]->stream), "cudaEventRecord");
    }
    pushed = true;
}

// One Ksp scan of the whole domain (Model::nucleate, 3S:752-759) over the slabs.
int SlabGroup::scan() {
    const int n = (int)m.size();
    sync_all();
    for (int s = 0; s < n; ++s) {
        on(s);
        push(s, false, halo);
        check_cuda(cudaEventRecord(ev_push[(size_t)s], m[(size_t)s]->stream), "cudaEventRecord");
    }
    pushed = true;
    for (int s = 0; s < n; ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        if (s > 0) check_cuda(cudaStreamWaitEvent(a.stream, ev_push[(size_t)s - 1], 0), "cudaStreamWaitEvent");
        if (s + 1 < n) check_cuda(cudaStreamWaitEvent(a.stream, ev_push[(size_t)s + 1], 0), "cudaStreamWaitEvent");
        a.kd.neta = a.neta;
        launch_ksp_candidates(a.kd, a.o_[a.cur], a.cr_[a.cur], a.p_[a.cur], a.kw, a.st, a.stream);
        a.launches += 3;
    }
    // nuclei whose stamp or exclusion marks reach slab s's stored planes
    auto near = [&](const std::vector<KspNucleus>& all, int s) {
        const Model& a = *m[(size_t)s];
        const int lo = a.x_off + 1, hi = a.x_off + a.g.nx, R = a.kd.box_half;
        std::vector<KspNucleus> r;
        for (const KspNucleus& q : all)
            if (q.x + R >= lo && q.x - R <= hi) r.push_back(q);
        return r;
    };
    std::vector<KspNucleus> accepted;
    std::vector<size_t> first((size_t)n + 1, 0);
    int nuclei = 0;
    for (int s = 0; s < n; ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        const std::vector<KspNucleus> pre = near(accepted, s);
        if ((int)pre.size() > cap) throw Error(NICR_ERR_STATE, "more nuclei near a slab in one Ksp scan than its list holds");
        if (!pre.empty())
            check_cuda(cudaMemcpyAsync(d_pre[(size_t)s], pre.data(), pre.size() * sizeof(KspNucleus),
                                       cudaMemcpyHostToDevice, a.stream), "H2D");
        launch_ksp_resolve_slab(a.kd, d_pre[(size_t)s], (int)pre.size(), d_out[(size_t)s], cap, a.o_[a.cur],
                                a.cr_[a.cur], a.p_[a.cur], a.eta_[a.ecur], a.kw, a.bud, a.kres, a.st, a.stream);
        a.launches += 1;
        KspResult r;
        check_cuda(cudaMemcpyAsync(&r, a.kres, sizeof r, cudaMemcpyDeviceToHost, a.stream), "D2H");
        a.sync();
        if (r.listed > cap) throw Error(NICR_ERR_STATE, "more nuclei in one Ksp scan of a slab than its list holds");
        first[(size_t)s] = accepted.size();
        accepted.resize(accepted.size() + (size_t)r.listed);
        if (r.listed)
            check_cuda(cudaMemcpy(accepted.data() + first[(size_t)s], d_out[(size_t)s], (size_t)r.listed * sizeof(KspNucleus),
                                  cudaMemcpyDeviceToHost), "D2H");
        nuclei += r.nuclei;
    }
    first[(size_t)n] = accepted.size();
    for (int s = 0; s + 1 < n; ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        const std::vector<KspNucleus> above(accepted.begin() + (long)first[(size_t)s + 1], accepted.end());
        const std::vector<KspNucleus> later = near(above, s);
        if (later.empty()) continue;
        if ((int)later.size() > cap) throw Error(NICR_ERR_STATE, "more nuclei near a slab in one Ksp scan than its list holds");
        check_cuda(cudaMemcpyAsync(d_pre[(size_t)s], later.data(), later.size() * sizeof(KspNucleus),
                                   cudaMemcpyHostToDevice, a.stream), "H2D");
        launch_ksp_apply(a.kd, d_pre[(size_t)s], (int)later.size(), a.o_[a.cur], a.cr_[a.cur], a.p_[a.cur],
                         a.eta_[a.ecur], a.kw, a.bud, a.kres, a.st, a.stream);
        a.launches += 1;
        a.sync();   // the host list must outlive the copy
    }
    for (auto& q : m)
        if (q->has_eta) q->eta_dirty = true;
    sync_all();
    check_cuda(cudaGetLastError(), "ksp");
    return nuclei;
}

int SlabGroup::advance(int nsteps, bool schedule, int* completed) {
    if (completed) *completed = 0;
    if (nsteps <= 0) return NICR_OK;
    const int n = (int)m.size();
    std::vector<Model::RunPlan> r((size_t)n);
    for (int s = 0; s < n; ++s) {
        on(s);
        m[(size_t)s]->run_begin(r[(size_t)s], nsteps, schedule);
    }
    int enqueued = 0;
    for (int i = 0; i < nsteps; ++i) {
        if (schedule) {
            // run()'s schedule (3S:1368-1372): a scan before the step whose time reaches the next nucleation time
            if (m[0]->ksp_due(r[0], i)) {
                if (any_failed()) break;   // a rejected step ends the batch; the rest would not run
                scan();
                for (auto& q : r) q.next += c.nucleation_period;
            }
            for (auto& q : r) q.sched[(size_t)i] = q.next;
        }
        one_step();
        ++enqueued;
    }
    int rc = NICR_OK, done = 0;
    err.clear();
    for (int s = 0; s < n; ++s) {
        on(s);
        r[(size_t)s].nsteps = enqueued;
        int d = 0;
        const int q = m[(size_t)s]->run_end(r[(size_t)s], &d);
        if (s == 0) { rc = q; done = d; }
        else if (q != rc || d != done) throw Error(NICR_ERR_STATE, "slabs disagree on the outcome of a step");
        if (q != NICR_OK && err.empty()) err = m[(size_t)s]->last_error;
    }
    if (completed) *completed = done;
    return rc;
}

int SlabGroup::nucleate(int* nuclei) {
    if (nuclei) *nuclei = 0;
    if (c.nucleation != NICR_NUC_KSP) return NICR_OK;
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        m[(size_t)s]->reset_status();
    }
    const int k = scan();
    if (nuclei) *nuclei = k;
    return NICR_OK;
}

void SlabGroup::get_field(int field, int index, double* host) {
    const long long plane_cells = (long long)c.ny * c.nz;
    for (int s = 0; s < (int)m.size(); ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        const double* d = a.field_ptr(field, index);
        a.copy_planes_out(d, host + (size_t)x0[(size_t)s] * plane_cells, a.sp.x_lo, a.sp.x_hi - a.sp.x_lo);
    }
}

void SlabGroup::set_field(int field, int index, const double* host) {
    const long long plane_cells = (long long)c.ny * c.nz;
    for (int s = 0; s < (int)m.size(); ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        // every stored plane, halos included, so the copies stay equal
        a.copy_planes_in(a.state_ptr(field, index), host + (size_t)a.x_off * plane_cells, 0, a.g.nx);
        a.eta_dirty = true;
    }
}

void SlabGroup::reset_inventory() {
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        m[(size_t)s]->reset_inventory();
    }
}

void SlabGroup::budget(nicr_budget* out) {
    *out = nicr_budget{};
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        nicr_budget b;
        m[(size_t)s]->budget(&b);
        double* dst[10] = {out->nucO, out->nucCr, out->ckO, out->ckCr, out->clipO, out->clipCr, out->bcO, out->bcCr,
                           out->initialO, out->initialCr};
        const double* src[10] = {b.nucO, b.nucCr, b.ckO, b.ckCr, b.clipO, b.clipCr, b.bcO, b.bcCr, b.initialO, b.initialCr};
        for (int q = 0; q < 10; ++q) put(dst[q], dd_add(dd(dst[q]), dd(src[q])));
        out->nuclei += b.nuclei;
        out->clipped += b.clipped;
    }
}

void SlabGroup::diagnostics(nicr_diagnostics* out) {
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        nicr_diagnostics d;
        m[(size_t)s]->diagnostics(&d);
        if (s == 0) { *out = d; continue; }
        double* dst[4] = {out->sum_O, out->sum_Cr, out->sum_phi, out->sum_h};
        const double* src[4] = {d.sum_O, d.sum_Cr, d.sum_phi, d.sum_h};
        for (int q = 0; q < 4; ++q) put(dst[q], dd_add(dd(dst[q]), dd(src[q])));
        out->min_O = pick_min(out->min_O, d.min_O); out->max_O = pick_max(out->max_O, d.max_O);
        out->min_Cr = pick_min(out->min_Cr, d.min_Cr); out->max_Cr = pick_max(out->max_Cr, d.max_Cr);
        out->min_Ni = pick_min(out->min_Ni, d.min_Ni);
        out->min_phi = pick_min(out->min_phi, d.min_phi); out->max_phi = pick_max(out->max_phi, d.max_phi);
    }
}

void SlabGroup::grain_stats(nicr_grain_stats* out, long long* cells, double* amount) {
    const int neta = m[0]->neta;
    std::vector<long long> cs((size_t)neta);
    std::vector<double> am((size_t)neta * 2);
    std::vector<long long> tc((size_t)neta, 0);
    std::vector<double> ta((size_t)neta * 2, 0.);
    for (int s = 0; s < (int)m.size(); ++s) {
        on(s);
        nicr_grain_stats g;
        m[(size_t)s]->grain_stats(&g, cs.data(), am.data());
        for (int q = 0; q < neta; ++q) {
            tc[(size_t)q] += cs[(size_t)q];
            put(&ta[2 * (size_t)q], dd_add(dd(&ta[2 * (size_t)q]), dd(&am[2 * (size_t)q])));
        }
        if (s == 0) { *out = g; continue; }
        out->min_eta = pick_min(out->min_eta, g.min_eta);
        out->max_eta = pick_max(out->max_eta, g.max_eta);
        out->min_s2 = pick_min(out->min_s2, g.min_s2);
        out->max_s2 = pick_max(out->max_s2, g.max_s2);
        put(out->sum_s2, dd_add(dd(out->sum_s2), dd(g.sum_s2)));
        put(out->mask, dd_add(dd(out->mask), dd(g.mask)));
        put(out->energy, dd_add(dd(out->energy), dd(g.energy)));
        out->gb_max = pick_max(out->gb_max, g.gb_max);
        out->unassigned += g.unassigned;
    }
    out->alive = 0;
    for (long long v : tc) out->alive += v > 0;
    if (cells) std::copy(tc.begin(), tc.end(), cells);
    if (amount) std::copy(ta.begin(), ta.end(), amount);
}

unsigned SlabGroup::vti_arrays(std::vector<unsigned char>& out, bool f64) {
    const size_t esz = f64 ? 8 : 4;
    const long long ny = c.ny, nz = c.nz, nx = c.nx, n = nx * ny * nz;
    out.resize(7 * (size_t)n * esz);
    unsigned range = 0;
    std::vector<unsigned char> part;
    for (int s = 0; s < (int)m.size(); ++s) {
        Model& a = *m[(size_t)s];
        on(s);
        a.refresh();
        a.ensure_mask();
        VtiArgs v{};
        v.g = a.own_grid();
        v.g.nstore = a.g.nstore;   // eta fields keep their stored stride
        const long long off = a.own_offset(), ns = v.g.ncells, nxs = v.g.nx;
        v.has_eta = a.has_eta ? 1 : 0;
        v.neta = a.neta;
        v.p = a.d_p() + off; v.o = a.d_o() + off; v.cr = a.d_cr() + off;
        v.muO = a.d_mu_o() + off; v.muCr = a.d_mu_cr() + off;
        v.gb = a.d_gb() + off;
        v.grain = a.grain_retained ? a.d_grain() + off : nullptr;
        v.eta = a.has_eta ? a.d_eta(0) + off : nullptr;
        if (!a.has_eta && !v.grain) throw Error(NICR_ERR_STATE, "grain map missing for grain_sum");
        void* d_out = nullptr;
        unsigned* d_range = nullptr;
        check_cuda(cudaMalloc(&d_out, 7 * (size_t)ns * esz), "cudaMalloc (VTI arrays)");
        check_cuda(cudaMalloc(&d_range, sizeof(unsigned)), "cudaMalloc");
        check_cuda(cudaMemsetAsync(d_range, 0, sizeof(unsigned), a.stream), "memset");
        launch_vti_arrays(v, d_out, f64, d_range, a.stream);
        part.resize(7 * (size_t)ns * esz);
        unsigned r = 0;
        check_cuda(cudaMemcpyAsync(part.data(), d_out, part.size(), cudaMemcpyDeviceToHost, a.stream), "D2H");
        check_cuda(cudaMemcpyAsync(&r, d_range, sizeof r, cudaMemcpyDeviceToHost, a.stream), "D2H");
        a.sync();
        cudaFree(d_out);
        cudaFree(d_range);
        check_cuda(cudaGetLastError(), "VTI arrays");
        range |= r;
        // the slab's X-fastest rows are the [x0, x1) pieces of the domain's rows
        for (int arr = 0; arr < 7; ++arr)
            for (long long row = 0; row < ny * nz; ++row)
                std::memcpy(out.data() + ((size_t)arr * n + (size_t)row * nx + x0[(size_t)s]) * esz,
                            part.data() + ((size_t)arr * ns + (size_t)row * nxs) * esz, (size_t)nxs * esz);
    }
    return range;
}

size_t SlabGroup::device_bytes() const {
    size_t b = 0;
    for (auto& q : m) b += q->device_bytes();
    return b;
}

}  // namespace nicr

// ------------------------------------------------------------------ C-ABI
struct nicr_slabs {
    std::unique_ptr<nicr::SlabGroup> g;
};

namespace {
std::string g_slabs_error;

template <class F>
int slabs_guarded(nicr_slabs* h, F&& f) {
    if (!h || !h->g) return NICR_ERR_INVALID_ARG;
    try {
        return f(*h->g);
    } catch (const nicr::Error& e) {
        h->g->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        h->g->err = "out of memory";
        return NICR_ERR_CUDA;
    } catch (const std::exception& e) {
        h->g->err = e.what();
        return NICR_ERR_CUDA;
    }
}
}  // namespace

// For nicr_slabs_write_vti, defined with the VTI writer (nicr_output.cpp)
nicr::SlabGroup* nicr_slabs_group(nicr_slabs* h) { return h ? h->g.get() : nullptr; }
void nicr_slabs_set_error(nicr_slabs* h, const std::string& e) {
    if (h && h->g) h->g->err = e;
}

extern "C" {

int nicr_slabs_create(const nicr_config* cfg, int nslabs, const int* devices, nicr_slabs** out) {
    if (!out) return NICR_ERR_INVALID_ARG;
    *out = nullptr;
    if (!cfg) {
        g_slabs_error = "no configuration";
        return NICR_ERR_INVALID_ARG;
    }
    try {
        auto* h = new nicr_slabs;
        try {
            h->g = std::make_unique<nicr::SlabGroup>(*cfg, nslabs, devices);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return NICR_OK;
    } catch (const nicr::Error& e) {
        g_slabs_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_slabs_error = e.what();
        return NICR_ERR_CUDA;
    }
}

void nicr_slabs_destroy(nicr_slabs* h) { delete h; }

int nicr_slabs_count(const nicr_slabs* h) { return h && h->g ? (int)h->g->m.size() : 0; }

int nicr_slabs_n_eta(const nicr_slabs* h) { return h && h->g ? h->g->m[0]->neta : 0; }

int nicr_slabs_info(const nicr_slabs* h, int slab, int* x0, int* x1, int* device, int* halo) {
    if (!h || !h->g || slab < 0 || slab >= (int)h->g->m.size()) return NICR_ERR_INVALID_ARG;
    if (x0) *x0 = h->g->x0[(size_t)slab];
    if (x1) *x1 = h->g->x1[(size_t)slab];
    if (device) *device = h->g->dev[(size_t)slab];
    if (halo) *halo = h->g->halo;
    return NICR_OK;
}

int nicr_slabs_step(nicr_slabs* h, int nsteps, int* completed) {
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { return g.advance(nsteps, false, completed); });
}

int nicr_slabs_run(nicr_slabs* h, int nsteps, int* completed) {
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { return g.advance(nsteps, true, completed); });
}

int nicr_slabs_nucleate(nicr_slabs* h, int* nuclei) {
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { return g.nucleate(nuclei); });
}

int nicr_slabs_get_field(nicr_slabs* h, int field, int index, double* host) {
    if (!host) return NICR_ERR_INVALID_ARG;
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { g.get_field(field, index, host); return NICR_OK; });
}

int nicr_slabs_set_field(nicr_slabs* h, int field, int index, const double* host) {
    if (!host) return NICR_ERR_INVALID_ARG;
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { g.set_field(field, index, host); return NICR_OK; });
}

int nicr_slabs_reset_inventory(nicr_slabs* h) {
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { g.reset_inventory(); return NICR_OK; });
}

int nicr_slabs_get_budget(nicr_slabs* h, nicr_budget* b) {
    if (!b) return NICR_ERR_INVALID_ARG;
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { g.budget(b); return NICR_OK; });
}

int nicr_slabs_get_diagnostics(nicr_slabs* h, nicr_diagnostics* d) {
    if (!d) return NICR_ERR_INVALID_ARG;
    return slabs_guarded(h, [&](nicr::SlabGroup& g) { g.diagnostics(d); return NICR_OK; });
}

int nicr_slabs_get_grain_stats(nicr_slabs* h, nicr_grain_stats* st, long long* cells, double* amount) {
    if (!st) return NICR_ERR_INVALID_ARG;
    return slabs_guarded(h, [&](nicr::SlabGroup& g) {
        if (!g.m[0]->has_eta) throw nicr::Error(NICR_ERR_STATE, "grain statistics exist only with evolving grains");
        g.grain_stats(st, cells, amount);
        return NICR_OK;
    });
}

long long nicr_slabs_steps_done(const nicr_slabs* h) { return h && h->g ? h->g->m[0]->steps_done : 0; }

long long nicr_slabs_kernel_launches(const nicr_slabs* h) { return h && h->g ? h->g->launches() : 0; }

void* nicr_slabs_stream(const nicr_slabs* h, int i) {
    if (!h || !h->g || i < 0 || i >= (int)h->g->m.size()) return nullptr;
    return static_cast<void*>(h->g->m[(size_t)i]->stream);
}

const char* nicr_slabs_last_error(const nicr_slabs* h) {
    return h && h->g ? h->g->err.c_str() : g_slabs_error.c_str();
}

}  // extern "C"
