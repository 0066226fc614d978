// Test infrastructure only: drives the UNMODIFIED reference solver so that its
// results can pin the C restatement (nicr_oracle.c) and serve as the timed CPU
// reference. Nothing in the product links or loads this program.
//
// Built by oracle/Makefile from the reference sources where they lie:
//   NICR_DIM=2 -> mpi2d/NiCr2D_grains.cpp
//   NICR_DIM=3 -> mpi3d-slab/NiCr3D_grains.cpp
// Same pattern as the reference's own mpi3d-slab/tests/regression_driver.cpp:1-8
// (rename main, include the solver translation unit, call Model directly).
//
// Usage: ref{2,3}d <reference CLI flags...> -- <command> [args] <command> ...
// Commands (executed in order):
//   inject FILE          packed interior doubles o,cr,p[,eta_1..eta_N] (X slowest)
//   reset_inventory      initialO/initialCr = current sums
//   step N               N raw Model::step() calls (stops on the first rejection)
//   run N                N steps on run()'s schedule (Ksp by physical time, 3S:1368-1385)
//   nucleate | refresh | invalidate
//   stamp X Y [Z]
//   scale_eta G I J [K] F  eta_G(I,J,K) *= F and invalidate the eta cache
//   scale_eta_if ...       the same, skipped when there is no eta_G
//   dump FILE            refresh + tagged binary dump of fields, budget and scalars
//   log FILE N           append Model::log and Model::grain_log rows for step N
//   vtk FILE | vti FILE | metadata
//   time_run N           like run N, printing wall seconds of the loop on rank 0
#define main nicr_reference_main
#if NICR_DIM == 2
#include "mpi2d/NiCr2D_grains.cpp"
#else
#include "mpi3d-slab/NiCr3D_grains.cpp"
#endif
#undef main
#include <chrono>
#include <cstdio>

namespace drv {

#if NICR_DIM == 2
#define AT(f, i, j, k) (f)(i, j)
#define KLOOP(m) for (int k = 1; k <= 1; ++k)
#else
#define AT(f, i, j, k) (f)(i, j, k)
#define KLOOP(m) for (int k = 1; k <= (m).c.nz; ++k)
#endif

static int nz_of(const Model& m) {
#if NICR_DIM == 2
    (void)m; return 1;
#else
    return m.c.nz;
#endif
}

struct Writer {
    std::ofstream f;
    explicit Writer(const std::string& path) : f(path, std::ios::binary) {
        if (!f) throw std::runtime_error("cannot write " + path);
        f.write("NICRDUMP", 8);
    }
    void header(const std::string& name, int kind, long long count) {
        char n[32] = {0};
        std::strncpy(n, name.c_str(), 31);
        f.write(n, 32);
        int k[2] = {kind, 0};
        f.write(reinterpret_cast<const char*>(k), 8);
        f.write(reinterpret_cast<const char*>(&count), 8);
    }
    void f64(const std::string& name, const std::vector<double>& v) {
        header(name, 1, (long long)v.size());
        f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 8));
    }
    void i64(const std::string& name, const std::vector<long long>& v) {
        header(name, 2, (long long)v.size());
        f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 8));
    }
    // long double as (hi, lo) double pairs: hi = (double)x, lo = (double)(x - hi)
    void ld(const std::string& name, const std::vector<long double>& v) {
        header(name, 3, (long long)v.size());
        for (long double x : v) {
            double hi = (double)x, lo = (double)(x - (long double)hi);
            f.write(reinterpret_cast<const char*>(&hi), 8);
            f.write(reinterpret_cast<const char*>(&lo), 8);
        }
    }
};

static std::vector<double> interior(const Model& m, const Field& a) {
    std::vector<double> v;
    if (a.a.empty()) return v;
    v.reserve((size_t)m.c.nx * m.c.ny * nz_of(m));
    for (int i = 1; i <= m.c.nx; ++i)
        for (int j = 1; j <= m.c.ny; ++j)
            KLOOP(m) v.push_back(AT(a, i, j, k));
    return v;
}

static void dump_model(Model& m, const std::string& path);

// Over several ranks (the thread-per-rank build) the state is first gathered
// into the root's snapshot model, as the reference's own output does
// (gather_state); the budget is then the ranks' reduced budget.
static void dump(Model& m, const std::string& path) {
    if (m.domain.size > 1) {
        m.gather_state();
        if (m.domain.rank == 0) dump_model(*m.snapshot, path);
        return;
    }
    dump_model(m, path);
}

static void dump_model(Model& m, const std::string& path) {
    m.refresh();
    Writer w(path);
    w.f64("o", interior(m, m.o));
    w.f64("cr", interior(m, m.cr));
    w.f64("p", interior(m, m.p));
    w.f64("muO", interior(m, m.muO));
    w.f64("muCr", interior(m, m.muCr));
    w.f64("mo", interior(m, m.mo));
    w.f64("mc", interior(m, m.mc));
    w.f64("gb", interior(m, m.gb));
    w.f64("grain", interior(m, m.grain));
    w.f64("eta_s2", interior(m, m.eta_s2));
#if NICR_DIM == 2
    w.f64("eta_pairs", interior(m, m.eta_pairs));
    w.f64("gb_initial", interior(m, m.gb_initial));
#endif
    for (size_t g = 0; g < m.eta.size(); ++g) w.f64("eta" + std::to_string(g + 1), interior(m, m.eta[g]));
    const Budget& b = m.b;
    w.ld("budget", {b.nucO, b.nucCr, b.ckO, b.ckCr, b.clipO, b.clipCr, b.bcO, b.bcCr});
    w.i64("counts", {b.nuclei, b.clipped});
    w.ld("initial", {m.initialO, m.initialCr});
    std::vector<double> seeds;
    for (auto& s : m.seeds) {
        seeds.push_back(s.x); seeds.push_back(s.y);
#if NICR_DIM == 3
        seeds.push_back(s.z);
#endif
    }
    w.f64("seeds", seeds);
#if NICR_DIM == 2
    std::vector<long long> vol(m.areas.begin(), m.areas.end());
#else
    std::vector<long long> vol(m.volumes.begin(), m.volumes.end());
#endif
    w.i64("volumes", vol);
    w.i64("center_seed_cells", {m.center_seed_cells});
    w.i64("n_eta", {(long long)m.eta.size()});
    if (!w.f) throw std::runtime_error("dump failed");
}

static void inject(Model& m, const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    const size_t n = (size_t)m.c.nx * m.c.ny * nz_of(m);
    std::vector<double> buf(n);
    auto load = [&](Field& a) {
        f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)(n * 8));
        if (!f) throw std::runtime_error("short inject file " + path);
        size_t q = 0;
        for (int i = 1; i <= m.c.nx; ++i)
            for (int j = 1; j <= m.c.ny; ++j)
                KLOOP(m) {
                    const double v = buf[q++];
                    if (i >= m.domain.first && i <= m.domain.last) AT(a, i, j, k) = v;
                }
    };
    load(m.o); load(m.cr); load(m.p);
    for (auto& e : m.eta) load(e);
#if NICR_DIM == 3
    m.invalidate_eta_cache();
#endif
    m.refresh();
}

static int run_steps(Model& m, int steps, double& next_nucleation, int& n_done, bool timed) {
    // run() schedule (2D:1219-1236, 3S:1368-1385) without output.
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 1; s <= steps; ++s) {
        const int n = n_done + 1;
        const double time = n * m.c.dt;
        if (m.c.nucleation == "ksp" && time + 1.e-12 * m.c.nucleation_period >= next_nucleation) {
            m.nucleate();
            next_nucleation += m.c.nucleation_period;
        }
        Budget before = m.b;
        try { m.step(); } catch (const std::exception& e) {
            m.b = before;
            if (m.domain.rank == 0) std::printf("REJECTED %d %s\n", n, e.what());
            return 1;
        }
        n_done = n;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (timed && m.domain.rank == 0)
        std::printf("TIME_RUN %d %.9f\n", steps, std::chrono::duration<double>(t1 - t0).count());
    return 0;
}

static int exercise(int argc, char** argv) {
    MPI_Init(&argc, &argv);
    int sep = argc;
    for (int q = 1; q < argc; ++q) if (std::string(argv[q]) == "--") { sep = q; break; }
    Config c = parse(sep, argv);
    Model m(c, MPI_COMM_WORLD);
    double next_nucleation = c.nucleation_period;
    int n_done = 0;
    std::ofstream logf, gdf, ghf;
    for (int q = sep + 1; q < argc; ++q) {
        const std::string cmd = argv[q];
        auto arg = [&](void) -> std::string {
            if (q + 1 >= argc) throw std::runtime_error("missing argument for " + cmd);
            return argv[++q];
        };
        if (cmd == "inject") inject(m, arg());
        else if (cmd == "reset_inventory") { m.initialO = Model::sum(m.o); m.initialCr = Model::sum(m.cr); }
        else if (cmd == "step") {
            const int n = std::stoi(arg());
            for (int s = 0; s < n; ++s) {
                // Budget rollback as run() does it (2D:1224-1225, 3S:1373-1374).
                Budget before = m.b;
                try { m.step(); ++n_done; } catch (const std::exception& e) {
                    m.b = before;
                    if (m.domain.rank == 0) std::printf("REJECTED %d %s\n", n_done + 1, e.what());
                    break;
                }
            }
        } else if (cmd == "run") run_steps(m, std::stoi(arg()), next_nucleation, n_done, false);
        else if (cmd == "time_run") run_steps(m, std::stoi(arg()), next_nucleation, n_done, true);
        else if (cmd == "nucleate") m.nucleate();
        else if (cmd == "refresh") m.refresh();
        else if (cmd == "invalidate") {
#if NICR_DIM == 3
            m.invalidate_eta_cache();
#endif
        } else if (cmd == "stamp") {
            const int x = std::stoi(arg()), y = std::stoi(arg());
#if NICR_DIM == 3
            const int z = std::stoi(arg());
            const int cells = m.stamp(x, y, z);
#else
            const int cells = m.stamp(x, y);
#endif
            if (m.domain.rank == 0) std::printf("STAMP %d\n", cells);
        } else if (cmd == "scale_eta_if") {
            // regression_driver.cpp:50-54: edit eta_G only when eta fields exist
            const int g = std::stoi(arg()), i = std::stoi(arg()), j = std::stoi(arg());
#if NICR_DIM == 3
            const int k = std::stoi(arg());
#endif
            const double fct = std::stod(arg());
            if ((size_t)g < m.eta.size()) {
                if (i >= m.domain.first && i <= m.domain.last) AT(m.eta[(size_t)g], i, j, k) *= fct;
#if NICR_DIM == 3
                m.invalidate_eta_cache();
#endif
            }
        } else if (cmd == "scale_eta") {
            const int g = std::stoi(arg()), i = std::stoi(arg()), j = std::stoi(arg());
#if NICR_DIM == 3
            const int k = std::stoi(arg());
#endif
            const double fct = std::stod(arg());
            if (i >= m.domain.first && i <= m.domain.last) AT(m.eta[(size_t)g], i, j, k) *= fct;
#if NICR_DIM == 3
            m.invalidate_eta_cache();
#endif
        } else if (cmd == "dump") dump(m, arg());
        else if (cmd == "log") {
            const std::string path = arg();
            const int n = std::stoi(arg());
            std::ofstream f(path, std::ios::app), gd(path + ".grain", std::ios::app), gh(path + ".history", std::ios::app);
            m.log(f, n);
            m.grain_log(gd, gh, n);
        } else if (cmd == "vtk") m.vtk(arg());
#if NICR_DIM == 3
        else if (cmd == "vti") m.vti(arg());
#endif
        else if (cmd == "metadata") m.metadata();
        else throw std::runtime_error("unknown driver command " + cmd);
    }
    MPI_Finalize();
    return 0;
}

}  // namespace drv

int main(int argc, char** argv) {
#ifdef NICR_MPI_THREAD_TEST
    // ref{2,3}d_threads RANKS <flags> -- <commands>
    if (argc < 2) return 1;
    const int np = std::stoi(argv[1]);
    return mpi_threads::run(np, [&] { return drv::exercise(argc - 1, argv + 1); });
#else
    try {
        return drv::exercise(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ERROR: %s\n", e.what());
        return 1;
    }
#endif
}
