// Output files and the solver program (host C++ over device data).
//   VTK legacy ASCII (2D:598-632, 3S:828-856), compressed VTI (3S:238-334,
//   3S:857-869), diagnostics.csv rows (2D:697-710, 3S:963-977), grain CSV rows
//   (2D:382-406, 3S:566-590), parameters.txt and grains.csv (2D:633-696,
//   3S:874-962), and run()/main() (2D:1161-1254, 3S:1309-1403).
// Formats (array names, column order, iostream precision 16/17, X-fastest
// order, the VTI block layout) follow the reference so that files written
// from bit-identical fields are byte-identical.
#include <zlib.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <locale>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nicr.h"
#include "nicr_model.h"
#include "nicr_slabs.h"


namespace fs = std::filesystem;

namespace {

using nicr::Model;

constexpr const char* VERSION2 = "mpi-eta-v1";
constexpr const char* VERSION3 = "mpi-eta-3d-xslab-optimized-v1";

long double ld(const double v[2]) { return (long double)v[0] + (long double)v[1]; }

// Host copies of the fields an output needs, in reference interior order.
struct Snapshot {
    const Model& m;
    long long n;
    std::vector<double> o, cr, p, gb, grain, muO, muCr, mo, mc, s2, pairs, gb_initial;
    std::vector<std::vector<double>> eta;
    explicit Snapshot(Model& mm, bool mu_m = true) : m(mm), n(mm.g.ncells) {
        mm.refresh();
        mm.ensure_mask();
        auto get = [&](int f, int idx, std::vector<double>& v) {
            v.resize((size_t)n);
            mm.get_field(f, idx, v.data());
        };
        get(NICR_FIELD_O, 0, o);
        get(NICR_FIELD_CR, 0, cr);
        get(NICR_FIELD_PHI, 0, p);
        get(NICR_FIELD_GB, 0, gb);
        if (mm.grain_retained) get(NICR_FIELD_GRAIN, 0, grain);
        if (mu_m) {
            muO.resize((size_t)n); muCr.resize((size_t)n); mo.resize((size_t)n); mc.resize((size_t)n);
            mm.fetch(mm.d_mu_o(), muO.data());
            mm.fetch(mm.d_mu_cr(), muCr.data());
            mm.fetch(mm.d_m_o(), mo.data());
            mm.fetch(mm.d_m_cr(), mc.data());
        }
        if (mm.has_eta) {
            get(NICR_FIELD_ETA_S2, 0, s2);
            eta.resize((size_t)mm.neta);
            for (int g = 0; g < mm.neta; ++g) get(NICR_FIELD_ETA, g, eta[(size_t)g]);
            if (mm.dim == 2) {
                get(NICR_FIELD_ETA_PAIRS, 0, pairs);
                get(NICR_FIELD_GB_INITIAL, 0, gb_initial);
            }
        } else if (mm.dim == 2) {
            get(NICR_FIELD_GB_INITIAL, 0, gb_initial);
        }
    }
    // current_grain (3S:527-533, 2D:360-366)
    int current_grain(long long q) const {
        if (p[q] >= .5) return 0;
        if (!m.has_eta) return int(grain[q]);
        double best = 1.e-12;
        int id = 0;
        for (size_t g = 0; g < eta.size(); ++g)
            if (eta[g][q] > best) { best = eta[g][q]; id = int(g) + 1; }
        return id;
    }
    // grain_sum (3S:534-545)
    double grain_sum(long long q) const {
        if (m.has_eta) {
            double value = 0.;
            for (size_t g = 0; g < eta.size(); ++g) value += double(g + 1) * eta[g][q];
            return value;
        }
        return grain[q] * (1. - nicr::h(p[q]));
    }
};

// ------------------------------------------------------------------ VTK
void write_vtk2(Model& m, const std::string& path) {
    Snapshot s(m);
    const auto& c = m.c;
    std::ofstream f(path);
    if (!f) throw nicr::Error(NICR_ERR_IO, "Cannot write " + path);
    f << std::setprecision(16) << "# vtk DataFile Version 3.0\n"
      << (m.has_eta ? "NiCr evolving metal grains; coordinates in metres\n" : "NiCr fixed-grain prototype; coordinates in metres\n")
      << "ASCII\nDATASET STRUCTURED_POINTS\n"
      << "DIMENSIONS " << c.nx << " " << c.ny << " 1\nORIGIN " << .5 * c.dx << " " << .5 * c.dy << " 0\nSPACING " << c.dx
      << " " << c.dy << " 1\nPOINT_DATA " << c.nx * c.ny << "\n";
    auto write = [&](const std::string& name, const std::function<double(long long)>& fn) {
        f << "SCALARS " << name << " double 1\nLOOKUP_TABLE default\n";
        for (int j = 1; j <= c.ny; ++j) {
            for (int i = 1; i <= c.nx; ++i) f << fn((long long)(i - 1) * c.ny + (j - 1)) << " ";
            f << "\n";
        }
    };
    write("phi", [&](long long q) { return s.p[q]; });
    write("conc_O", [&](long long q) { return s.o[q]; });
    write("conc_Cr", [&](long long q) { return s.cr[q]; });
    write("conc_Ni", [&](long long q) { return 1. - s.o[q] - s.cr[q]; });
    write("grain_id", [&](long long q) { return m.has_eta ? double(s.current_grain(q)) : s.grain[q]; });
    write("GB_mask", [&](long long q) { return s.gb[q]; });
    write("GB_active", [&](long long q) { return (1. - nicr::h(s.p[q])) * s.gb[q]; });
    write("mu_O", [&](long long q) { return s.muO[q]; });
    write("mu_Cr", [&](long long q) { return s.muCr[q]; });
    write("M_O", [&](long long q) { return s.mo[q]; });
    write("M_Cr", [&](long long q) { return s.mc[q]; });
    if (m.has_eta) {
        write("grain_id_initial", [&](long long q) { return s.grain[q]; });
        write("GB_initial", [&](long long q) { return s.gb_initial[q]; });
        write("GB_eta_indicator", [&](long long q) { return std::min(1., 16. * s.pairs[q]); });
        write("metal_fraction", [&](long long q) { return 1. - nicr::h(s.p[q]); });
        write("eta_sum_sq", [&](long long q) { return s.s2[q]; });
        write("active_grain_id", [&](long long q) { return double(s.current_grain(q)); });
        if (c.eta_output_all)
            for (size_t g = 0; g < s.eta.size(); ++g)
                write("eta_" + std::to_string(g + 1), [&](long long q) { return s.eta[g][q]; });
    }
    if (!f) throw nicr::Error(NICR_ERR_IO, "Output write failed: " + path);
}

// X-fastest traversal of a 3D domain stored X-slowest
template <class Fn>
void for_x_fastest(const nicr_config& c, Fn fn) {
    for (int k = 1; k <= c.nz; ++k)
        for (int j = 1; j <= c.ny; ++j)
            for (int i = 1; i <= c.nx; ++i) fn(((long long)(i - 1) * c.ny + (j - 1)) * c.nz + (k - 1), i == c.nx);
}

std::array<std::function<double(long long)>, 7> arrays3(const Snapshot& s) {
    return {[&](long long q) { return s.p[q]; }, [&](long long q) { return s.o[q]; },
            [&](long long q) { return s.cr[q]; }, [&](long long q) { return s.muO[q]; },
            [&](long long q) { return s.muCr[q]; }, [&](long long q) { return s.grain_sum(q); },
            [&](long long q) { return s.gb[q]; }};
}
constexpr std::array<const char*, 7> NAMES3 = {"phi", "conc_O", "conc_Cr", "mu_O", "mu_Cr", "grain_sum", "GB_mask"};

void write_vtk3(Model& m, const std::string& path) {
    Snapshot s(m);
    const auto& c = m.c;
    std::ofstream f(path);
    if (!f) throw nicr::Error(NICR_ERR_IO, "Cannot write " + path);
    f << std::setprecision(17) << "# vtk DataFile Version 3.0\nNiCr 3D oxidation and metal grains; metres\n"
      << "ASCII\nDATASET STRUCTURED_POINTS\nDIMENSIONS " << c.nx << " " << c.ny << " " << c.nz << "\nORIGIN "
      << .5 * c.dx << " " << .5 * c.dy << " " << .5 * c.dz << "\nSPACING " << c.dx << " " << c.dy << " " << c.dz
      << "\nPOINT_DATA " << c.nx * c.ny * c.nz << "\n";
    const auto fns = arrays3(s);
    for (size_t a = 0; a < NAMES3.size(); ++a) {
        f << "SCALARS " << NAMES3[a] << " double 1\nLOOKUP_TABLE default\n";
        for_x_fastest(c, [&](long long q, bool last) {
            f << fns[a](q) << " ";
            if (last) f << "\n";
        });
    }
    if (!f) throw nicr::Error(NICR_ERR_IO, "Output write failed: " + path);
}

// ------------------------------------------------------------------ VTI
// VTK XML ImageData, raw appended data, zlib blocks of 64 KiB with UInt64
// headers (block count, block size, last block size, compressed sizes),
// written to path.tmp and renamed on success (write_vti, 3S:238-334). The
// arrays arrive in file order and type from the GPU (launch_vti_arrays); the
// blocks are independent zlib streams, compressed here by a pool of host
// threads, so the file is the same byte for byte as a serial writer's.
constexpr std::uint64_t kVtiBlock = 65536;

void put_u64(std::string& s, std::uint64_t v) {
    for (int q = 0; q < 8; ++q) s.push_back((char)(unsigned char)(v >> (8 * q)));
}

void compose_vti(const nicr_config& c, const unsigned char* arrays, bool f64, const std::string& path) {
    const std::uint64_t esz = f64 ? 8 : 4;
    const std::uint64_t n = std::uint64_t(c.nx) * c.ny * c.nz, total = n * esz;
    const std::uint64_t nb = (total + kVtiBlock - 1) / kVtiBlock;
    const size_t narr = NAMES3.size(), jobs = narr * (size_t)nb;
    std::vector<std::vector<unsigned char>> blocks(jobs);
    std::atomic<size_t> next{0};
    std::atomic<int> zrc{Z_OK};
    auto work = [&] {
        for (size_t b; (b = next.fetch_add(1)) < jobs;) {
            const size_t arr = b / (size_t)nb;
            const std::uint64_t bi = b % nb, off = bi * kVtiBlock;
            const std::uint64_t len = std::min<std::uint64_t>(kVtiBlock, total - off);
            std::vector<unsigned char>& dst = blocks[b];
            dst.resize((size_t)compressBound((uLong)len));
            uLongf dlen = (uLongf)dst.size();
            const int rc = compress2(dst.data(), &dlen, arrays + arr * total + off, (uLong)len, c.compression_level);
            if (rc != Z_OK) zrc = rc;
            dst.resize(dlen);
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nthreads = std::min<size_t>(jobs, std::max(1u, std::min(hw, 32u)));
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (zrc != Z_OK) throw nicr::Error(NICR_ERR_IO, "zlib compression failed: " + std::to_string(zrc.load()));

    std::vector<std::uint64_t> offset(narr);
    std::uint64_t run = 0;
    for (size_t arr = 0; arr < narr; ++arr) {
        offset[arr] = run;
        run += 24 + 8 * nb;
        for (std::uint64_t bi = 0; bi < nb; ++bi) run += blocks[arr * (size_t)nb + (size_t)bi].size();
    }
    std::ostringstream h;
    h.imbue(std::locale::classic());
    h << std::setprecision(17) << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\" compressor=\"vtkZLibDataCompressor\">\n"
      << " <ImageData WholeExtent=\"0 " << c.nx - 1 << " 0 " << c.ny - 1 << " 0 " << c.nz - 1 << "\" Origin=\""
      << .5 * c.dx << " " << .5 * c.dy << " " << .5 * c.dz << "\" Spacing=\"" << c.dx << " " << c.dy << " " << c.dz
      << "\">\n  <Piece Extent=\"0 " << c.nx - 1 << " 0 " << c.ny - 1 << " 0 " << c.nz - 1 << "\">\n"
      << "   <PointData Scalars=\"phi\">\n";
    for (size_t arr = 0; arr < narr; ++arr)
        h << "    <DataArray type=\"" << (f64 ? "Float64" : "Float32") << "\" Name=\"" << NAMES3[arr]
          << "\" NumberOfComponents=\"1\" format=\"appended\" offset=\"" << std::setw(20) << std::setfill('0')
          << offset[arr] << std::setfill(' ') << "\"/>\n";
    h << "   </PointData>\n   <CellData/>\n  </Piece>\n </ImageData>\n <AppendedData encoding=\"raw\">\n_";

    const std::string temp = path + ".tmp";
    std::ofstream f(temp, std::ios::binary | std::ios::trunc);
    if (!f) throw nicr::Error(NICR_ERR_IO, "Cannot open " + temp);
    auto fail = [&] {
        f.close();
        std::error_code ec;
        fs::remove(temp, ec);
        throw nicr::Error(NICR_ERR_IO, "VTI write failed (check storage/quota): " + temp);
    };
    const std::string head = h.str();
    f.write(head.data(), (std::streamsize)head.size());
    for (size_t arr = 0; arr < narr; ++arr) {
        std::string bh;
        put_u64(bh, nb);
        put_u64(bh, kVtiBlock);
        put_u64(bh, total % kVtiBlock);
        for (std::uint64_t bi = 0; bi < nb; ++bi) put_u64(bh, blocks[arr * (size_t)nb + (size_t)bi].size());
        f.write(bh.data(), (std::streamsize)bh.size());
        for (std::uint64_t bi = 0; bi < nb; ++bi) {
            const auto& blk = blocks[arr * (size_t)nb + (size_t)bi];
            f.write(reinterpret_cast<const char*>(blk.data()), (std::streamsize)blk.size());
        }
        if (!f) fail();
    }
    f << "\n </AppendedData>\n</VTKFile>\n";
    f.flush();
    if (!f) fail();
    f.close();
    if (!f) fail();
    fs::rename(temp, path);
}

// Asynchronous VTI writer of one model. submit() enqueues, on the model's
// stream, the refresh of mu/M, the kernel that builds the frame's arrays in a
// device staging buffer, and (on a copy stream, after an event) their copy to
// pinned host memory; a host thread then waits for the copy, compresses and
// writes the file while the model keeps stepping. One frame is in flight at a
// time: submit() and wait() first finish the previous one and report its
// error, if any.
class AsyncVti {
    int device = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t ready = nullptr, copied = nullptr;
    void* d_stage = nullptr;
    unsigned char* h_stage = nullptr;
    unsigned* d_range = nullptr;
    unsigned* h_range = nullptr;
    size_t bytes = 0;
    std::thread worker;
    std::string error;
    int error_code = NICR_OK;

    void release_buffers() {
        if (d_stage) cudaFree(d_stage);
        if (h_stage) cudaFreeHost(h_stage);
        d_stage = nullptr;
        h_stage = nullptr;
        bytes = 0;
    }

public:
    explicit AsyncVti(int dev) : device(dev) {
        nicr::check_cuda(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking), "cudaStreamCreate");
        nicr::check_cuda(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "cudaEventCreate");
        nicr::check_cuda(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming), "cudaEventCreate");
        nicr::check_cuda(cudaMalloc(&d_range, sizeof(unsigned)), "cudaMalloc");
        nicr::check_cuda(cudaMallocHost(&h_range, sizeof(unsigned)), "cudaMallocHost");
    }
    ~AsyncVti() {
        finish();
        cudaSetDevice(device);
        release_buffers();
        if (d_range) cudaFree(d_range);
        if (h_range) cudaFreeHost(h_range);
        if (ready) cudaEventDestroy(ready);
        if (copied) cudaEventDestroy(copied);
        if (copy) cudaStreamDestroy(copy);
    }
    // joins the writer thread; returns (and clears) the error of the last frame
    int finish(std::string* msg = nullptr) {
        if (worker.joinable()) worker.join();
        const int rc = error_code;
        if (msg) *msg = error;
        error_code = NICR_OK;
        error.clear();
        return rc;
    }
    void submit(Model& m, const std::string& path) {
        std::string msg;
        const int rc = finish(&msg);
        if (rc != NICR_OK) throw nicr::Error(rc, msg);
        const nicr_config c = m.c;
        const bool f64 = c.output_float64 != 0;
        const size_t need = NAMES3.size() * (size_t)m.g.ncells * (f64 ? 8 : 4);
        if (need != bytes) {
            release_buffers();
            nicr::check_cuda(cudaMalloc(&d_stage, need), "cudaMalloc (VTI staging)");
            nicr::check_cuda(cudaMallocHost(&h_stage, need), "cudaMallocHost (VTI staging)");
            bytes = need;
        }
        m.refresh();
        m.ensure_mask();
        nicr::VtiArgs a{};
        a.g = m.g;
        a.has_eta = m.has_eta ? 1 : 0;
        a.neta = m.neta;
        a.p = m.d_p(); a.o = m.d_o(); a.cr = m.d_cr();
        a.muO = m.d_mu_o(); a.muCr = m.d_mu_cr();
        a.gb = m.d_gb();
        a.grain = m.grain_retained ? m.d_grain() : nullptr;
        a.eta = m.has_eta ? m.d_eta(0) : nullptr;
        if (!m.has_eta && !a.grain) throw nicr::Error(NICR_ERR_STATE, "grain map missing for grain_sum");
        nicr::check_cuda(cudaMemsetAsync(d_range, 0, sizeof(unsigned), m.stream), "memset");
        nicr::launch_vti_arrays(a, d_stage, f64, d_range, m.stream);
        nicr::check_cuda(cudaGetLastError(), "VTI arrays");
        nicr::check_cuda(cudaEventRecord(ready, m.stream), "cudaEventRecord");
        nicr::check_cuda(cudaStreamWaitEvent(copy, ready, 0), "cudaStreamWaitEvent");
        nicr::check_cuda(cudaMemcpyAsync(h_stage, d_stage, bytes, cudaMemcpyDeviceToHost, copy), "D2H");
        nicr::check_cuda(cudaMemcpyAsync(h_range, d_range, sizeof(unsigned), cudaMemcpyDeviceToHost, copy), "D2H");
        nicr::check_cuda(cudaEventRecord(copied, copy), "cudaEventRecord");
        worker = std::thread([this, c, f64, path] {
            try {
                cudaSetDevice(device);
                nicr::check_cuda(cudaEventSynchronize(copied), "VTI copy");
                const unsigned r = *h_range;
                if (r) {
                    int arr = 0;
                    while (!(r & (1u << arr))) ++arr;
                    throw nicr::Error(NICR_ERR_IO, std::string("VTI ") + NAMES3[(size_t)arr] +
                                                       " exceeds output type range; use --output-precision float64.");
                }
                compose_vti(c, h_stage, f64, path);
            } catch (const nicr::Error& e) {
                error_code = e.code;
                error = e.what();
            } catch (const std::exception& e) {
                error_code = NICR_ERR_IO;
                error = e.what();
            }
        });
    }
};

AsyncVti& vti_writer(Model& m) {
    if (!m.output_writer) m.output_writer = std::make_shared<AsyncVti>(m.c.device);
    return *static_cast<AsyncVti*>(m.output_writer.get());
}

void write_vti3_async(Model& m, const std::string& path) { vti_writer(m).submit(m, path); }

void output_wait(Model& m) {
    if (!m.output_writer) return;
    std::string msg;
    const int rc = static_cast<AsyncVti*>(m.output_writer.get())->finish(&msg);
    if (rc != NICR_OK) throw nicr::Error(rc, msg);
}

void write_vti3(Model& m, const std::string& path) {
    write_vti3_async(m, path);
    output_wait(m);
}

// One output frame. With `async`, a 3D VTI frame is finished by the model's
// writer thread while stepping continues (output_wait joins it); the ASCII
// VTK frames are written at once.
void write_visualization(Model& m, const std::string& stem, bool async = false) {
    if (m.dim == 2) write_vtk2(m, stem + ".vtk");
    else if (m.c.output_vti) {
        if (async) write_vti3_async(m, stem + ".vti");
        else write_vti3(m, stem + ".vti");
    } else write_vtk3(m, stem + ".vtk");
}

// ------------------------------------------------------------------ CSV rows
// One diagnostics.csv row from the diagnostics and budget values (3S:963-977)
std::string log_row(const nicr_config& c, int dim, const nicr_diagnostics& d, const nicr_budget& b, int n) {
    const long double so = ld(d.sum_O), sc = ld(d.sum_Cr), po = ld(d.sum_phi), sumH = ld(d.sum_h);
    const long double ro = so - ld(b.initialO) - ld(b.bcO) - ld(b.nucO) - ld(b.ckO) - ld(b.clipO);
    const long double rc = sc - ld(b.initialCr) - ld(b.bcCr) - ld(b.nucCr) - ld(b.ckCr) - ld(b.clipCr);
    const int cells = dim == 3 ? c.nx * c.ny * c.nz : c.nx * c.ny;
    std::ostringstream f;
    f << std::setprecision(17) << n << "," << n * c.dt << "," << so << "," << sc << "," << po / cells << ","
      << ld(b.bcO) << "," << ld(b.nucO) << "," << ld(b.nucCr) << "," << ld(b.ckO) << "," << ld(b.ckCr) << ","
      << ld(b.clipO) << "," << ld(b.clipCr) << "," << ro << "," << rc << "," << b.nuclei << "," << b.clipped << ","
      << d.min_O << "," << d.max_O << "," << d.min_Cr << "," << d.max_Cr << "," << d.min_Ni << "," << d.min_phi << ","
      << d.max_phi;
    if (dim == 3) f << "," << sumH / cells << "," << sumH * c.dx * c.dy * c.dz;
    f << "\n";
    return f.str();
}

std::string log_row(Model& m, int n) {
    nicr_diagnostics d;
    m.diagnostics(&d);
    nicr_budget b;
    m.budget(&b);
    return log_row(m.c, m.dim, d, b, n);
}

// grain_diagnostics.csv and grain_history.csv rows from the grain statistics
// (Model::grain_log, 3S:566-590)
void grain_rows(const nicr_config& c, int dim, int neta, const nicr_grain_stats& s, const std::vector<long long>& cells,
                const std::vector<double>& amount, int n, std::string& diag, std::string& history) {
    const int ncell = dim == 3 ? c.nx * c.ny * c.nz : c.nx * c.ny;
    std::ostringstream f, h;
    f << std::setprecision(17) << n << "," << n * c.dt << "," << s.min_eta << "," << s.max_eta << "," << s.min_s2 << ","
      << s.max_s2 << "," << ld(s.sum_s2) / ncell << "," << s.alive << "," << s.unassigned << ",";
    if (dim == 3) f << ld(s.mask) * c.dx * c.dy * c.dz;
    else f << ld(s.mask) * c.dx * c.dy;
    f << "," << s.gb_max << "," << ld(s.energy) << "\n";
    for (int g = 0; g < neta; ++g) {
        const long double a = (long double)amount[2 * g] + (long double)amount[2 * g + 1];
        h << std::setprecision(17) << n << "," << n * c.dt << "," << g + 1 << "," << cells[(size_t)g] << "," << a << ",";
        if (dim == 3) h << a * c.dx * c.dy * c.dz;
        else h << a * c.dx * c.dy;
        h << "\n";
    }
    diag = f.str();
    history = h.str();
}

void grain_rows(Model& m, int n, std::string& diag, std::string& history) {
    diag.clear();
    history.clear();
    if (!m.has_eta) return;
    nicr_grain_stats s;
    std::vector<long long> cells((size_t)m.neta);
    std::vector<double> amount((size_t)m.neta * 2);
    m.grain_stats(&s, cells.data(), amount.data());
    grain_rows(m.c, m.dim, m.neta, s, cells, amount, n, diag, history);
}

// ------------------------------------------------------------------ metadata
// What parameters.txt and grains.csv need of a domain (a Model, or a slab
// group's totals).
struct MetaView {
    nicr_config c;
    nicr::EtaCoef ec;
    int dim = 3;
    bool has_eta = false;
    int neta = 0;
    int center_seed_cells = 0;
    std::vector<double> seeds;
    std::vector<long long> volumes;
    size_t bytes = 0;
    std::string backend = "execution_backend=cuda_sm100a_single_gpu\n";
    size_t device_bytes() const { return bytes; }
};

MetaView meta_of(const Model& m) {
    MetaView v;
    v.c = m.c; v.ec = m.ec; v.dim = m.dim; v.has_eta = m.has_eta; v.neta = m.neta;
    v.center_seed_cells = m.center_seed_cells; v.seeds = m.seeds; v.volumes = m.volumes; v.bytes = m.device_bytes();
    return v;
}

MetaView meta_of(const nicr::SlabGroup& g) {
    MetaView v = meta_of(*g.m[0]);
    v.center_seed_cells = 0;
    std::fill(v.volumes.begin(), v.volumes.end(), 0);
    for (auto& q : g.m) {
        v.center_seed_cells += q->center_seed_cells;
        for (size_t k = 0; k < v.volumes.size(); ++k) v.volumes[k] += q->volumes[k];
    }
    v.bytes = g.device_bytes();
    v.backend = "execution_backend=cuda_sm100a_x_slabs_" + std::to_string(g.m.size()) + "\n";
    return v;
}

void metadata(const MetaView& m, const std::string& out) {
    const auto& c = m.c;
    const nicr::EtaCoef ec = m.ec;
    const double pi = nicr::PI;
    const std::string& backend = m.backend;
    std::ofstream f(out + "/parameters.txt");
    auto onoff = [](bool b) { return b ? "on" : "off"; };
    const char* bc = c.bc == NICR_BC_MU ? "mu" : c.bc == NICR_BC_CLOSED ? "closed" : "concentration";
    const char* ck = c.ck == NICR_CK_OFF ? "off" : "legacy";
    const char* bounds = c.bounds == NICR_BOUNDS_LEGACY ? "legacy" : "stop";
    const char* nuc = c.nucleation == NICR_NUC_CENTER ? "center" : c.nucleation == NICR_NUC_OFF ? "off" : "ksp";
    const std::string eta_output = c.eta_output_all ? "all" : "summary";
    if (m.dim == 2) {
        f << std::setprecision(17)
          << (m.has_eta ? "STATUS: COUPLED ETA/OXIDATION MODEL; GRAIN PARAMETERS REQUIRE CALIBRATION\n"
                        : "STATUS: UNCALIBRATED FIXED-GRAIN TRANSPORT PROTOTYPE\n")
          << "nx=" << c.nx << "\nny=" << c.ny << "\ndx_m=" << c.dx << "\ndy_m=" << c.dy << "\ndt_s=" << c.dt
          << "\nsteps=" << c.steps << "\noxygen_bc=" << bc << "\nCk=" << ck << "\nbounds=" << bounds
          << "\nmpi_processes=1\nmpi_decomposition=X slabs"
          << "\nversion=" << VERSION2 << "\nnucleation_mode=" << nuc
          << "\ninitial_center_seed_cells=" << m.center_seed_cells << "\ngrain_structure=" << onoff(c.grains)
          << "\noxygen_diffusion=" << onoff(c.oxygen_diffusion)
          << "\noxygen_boundary_supply=" << (c.oxygen_diffusion ? bc : "disabled") << "\nW=" << nicr::Phys::W
          << "\nkappa_phi=" << nicr::Phys::kp << "\nL_phi=" << nicr::Phys::L << "\nmu_res_model_units=" << c.mu_res
          << "\nsurface_mobility_concentration_reference=" << c.surface_c_ref
          << "\nleft_edge_sites_requested=" << c.left_edge_sites
          << "\nleft_edge_sites_active=" << (c.grains ? c.left_edge_sites : 0)
          << "\ngrain_diameter_target_grid=" << c.grain_diameter_grid
          << "\ngrain_diameter_target_m=" << c.grain_diameter_grid * c.dx << "\nvoronoi_sites=" << m.seeds.size() / 2
          << "\ngb_mask_FWHM_grid=" << c.gb_fwhm_grid << "\ngb_mask_FWHM_m=" << c.gb_fwhm_grid * c.dx
          << "\ngb_mask_integral_effective_width_grid=" << c.gb_fwhm_grid * std::sqrt(pi) / (2. * std::sqrt(std::log(2.)))
          << "\ngb_mask_integral_effective_width_m=" << c.gb_fwhm_grid * c.dx * std::sqrt(pi) / (2. * std::sqrt(std::log(2.)))
          << "\ngb_peak_mobility_factor_O=" << c.gb_factor_o << "\ngb_peak_mobility_factor_Cr=" << c.gb_factor_cr
          << "\nrandom_seed=" << c.random_seed << "\nnucleus_geometric_radius_grid=" << c.radius_grid
          << "\nnucleus_geometric_radius_m=" << c.radius_grid * c.dx << "\nnucleation_period_s=" << c.nucleation_period
          << "\nNOTE: Vm=1 is retained, not evidence that energy/mobility units have been physically audited.\n"
          << "NOTE: no GB migration, GB energy, segregation, oxide GBs, or interphase enhancement.\n"
          << "NOTE: cell-centred grid; periodic Y; no-flux right; natural concentration/phi derivatives in X.\n";
        f << backend;
        f << "grain_evolution_requested=" << onoff(c.grain_evolution) << "\ngrain_evolution_active=" << onoff(m.has_eta) << "\n";
        if (m.has_eta) {
            f << "eta_fields=" << m.neta << "\neta_W=" << c.eta_W << "\neta_kappa=" << ec.K << "\neta_L=" << c.eta_L
              << "\neta_oxide_penalty=" << ec.A << "\neta_width_10_90_grid=" << 2. * std::log(9.) * ec.ell / c.dx
              << "\neta_mask_integrated_width_m=" << 8. * ec.ell / 3. << "\neta_transport_scale=" << ec.scale
              << "\neta_planar_GB_energy_model_units=" << std::sqrt(2. * ec.K * c.eta_W) / 3.
              << "\neta_planar_geometric_mobility_model_units=" << 3. * c.eta_L * ec.ell << "\neta_output=" << eta_output
              << "\nNOTE: New grain coefficients are provisional, not experimental Ni-Cr calibration.\n"
              << "NOTE: Dynamic eta modifies the GB pathways AND adds the reciprocal grain-energy force to phi.\n"
              << "NOTE: GB factors refer to the original integrated-width convention; GB_mask includes eta_transport_scale.\n";
        } else
            f << "NOTE: fixed initial grain map and Gaussian GB mask.\n";
        if (c.nucleation == NICR_NUC_CENTER)
            f << "initial_oxide_center_x_m=" << 0.5 * c.nx * c.dx << "\ninitial_oxide_center_y_m=" << 0.5 * c.ny * c.dy
              << "\ninitial_oxide_center_i=" << 0.5 * (double(c.nx) + 1.) << "\ninitial_oxide_center_j="
              << 0.5 * (double(c.ny) + 1.)
              << "\nNOTE: one initial hard oxide only; no later Ksp insertion or replacement seed.\n";
        if (!c.grains) f << "NOTE: single grain; grain_id=1 and GB_mask=0; configured GB factors are inactive.\n";
        if (!c.oxygen_diffusion)
            f << "NOTE: O transport and continuing O boundary supply are off; initial inventory, hard seed assignments, optional Ck and bounds treatment remain.\n";
        std::ofstream g(out + "/grains.csv");
        g << "grain_id,seed_x_grid,seed_y_grid,area_cells,equivalent_diameter_grid,equivalent_diameter_m\n";
        long double mean = 0;
        const size_t ng = m.volumes.size();
        for (size_t k = 0; k < ng; ++k) {
            const double d = 2. * std::sqrt(m.volumes[k] / pi);
            mean += d;
            g << std::setprecision(17) << k + 1 << "," << m.seeds[2 * k] << "," << m.seeds[2 * k + 1] << ","
              << m.volumes[k] << "," << d << "," << d * c.dx << "\n";
        }
        mean /= ng;
        f << "measured_arithmetic_mean_equivalent_diameter_grid=" << mean << "\n";
        if (!f || !g) throw nicr::Error(NICR_ERR_IO, "Metadata write failed.");
        return;
    }
    const std::string fmt = c.output_vti ? "vti" : "vtk";
    const std::string prec = c.output_float64 ? "float64" : "float32";
    f << std::setprecision(17) << "model=NiCr_3D_oxidation_metal_grains\nversion=" << VERSION3 << "\nnx=" << c.nx
      << "\nny=" << c.ny << "\nnz=" << c.nz << "\ndx_m=" << c.dx << "\ndy_m=" << c.dy << "\ndz_m=" << c.dz
      << "\ndt_s=" << c.dt << "\nsteps=" << c.steps << "\noutput_every=" << c.output_every
      << "\nvtk_fields=phi,conc_O,conc_Cr,mu_O,mu_Cr,grain_sum,GB_mask"
      << "\noutput_format=" << fmt
      << "\noutput_precision=" << (fmt == "vtk" ? std::string("float64_ascii_17digits") : prec)
      << "\noutput_compression=" << (fmt == "vti" ? "zlib_raw_appended" : "none")
      << "\ncompression_level=" << c.compression_level << "\nfrozen_eta_cache=" << onoff(c.frozen_eta_cache)
      << "\nnucleation_search=bounded_periodic_neighborhoods_original_order_and_predicates"
      << "\nGB_mask_definition="
      << (!c.grains ? "zero;single_crystal"
                    : (m.has_eta ? "eta_transport_scale*min(1,16*sum_(a<b) eta_a^2*eta_b^2);no_extra_phi_mask"
                                 : "exp(-4*ln(2)*distance_to_GB_grid^2/gb_fwhm_grid^2);fixed_Voronoi;zero_when_one_grain;no_extra_phi_mask"))
      << "\ngrain_sum_definition="
      << (m.has_eta ? "sum_(g=1..N) g*eta_g;unnormalized;no_extra_phi_mask" : "initial_grain_id*(1-h(phi));fixed_grain_fallback_no_eta_fields")
      << "\noxygen_bc=" << bc << "\nCk=" << ck << "\nbounds=" << bounds
      << "\nmpi_processes=1\nmpi_decomposition=X_slabs_YZ_planes"
      << "\ntransverse_bc=periodic_Y_and_Z\nright_bc=no_flux"
      << "\nnucleation_mode=" << nuc << "\ninitial_center_seed_cells=" << m.center_seed_cells
      << "\ngrain_structure=" << onoff(c.grains) << "\ngrain_evolution_requested=" << onoff(c.grain_evolution)
      << "\ngrain_evolution_active=" << onoff(m.has_eta) << "\noxygen_diffusion=" << onoff(c.oxygen_diffusion)
      << "\noxygen_boundary_supply=" << (c.oxygen_diffusion ? bc : "disabled")
      << "\nVm=" << 1. << "\nW=" << nicr::Phys::W << "\nkappa_phi=" << nicr::Phys::kp << "\nL_phi=" << nicr::Phys::L
      << "\nkappa_O=" << nicr::Phys::ko << "\nkappa_Cr=" << nicr::Phys::kc
      << "\nmatrix_mobility_prefactor_O=" << nicr::Phys::bmo << "\nmatrix_mobility_prefactor_Cr=" << nicr::Phys::bmc
      << "\noxide_mobility_prefactor_O=" << nicr::Phys::boo << "\noxide_mobility_prefactor_Cr=" << nicr::Phys::boc
      << "\nbulk_O=" << nicr::Phys::bulkO << "\nbulk_Cr=" << c.bulk_cr << "\nlayer_O=" << c.layer_o
      << "\nlayer_Cr=" << nicr::Phys::layerCr << "\noxide_O=" << nicr::Phys::oxideO << "\noxide_Cr=" << nicr::Phys::oxideCr
      << "\nCk_O=" << nicr::Phys::ckO << "\nCk_Cr=" << nicr::Phys::ckCr << "\nKsp=" << c.ksp
      << "\nmu_res_model_units=" << c.mu_res << "\nsurface_mobility_concentration_reference=" << c.surface_c_ref
      << "\nleft_face_sites_requested=" << c.left_edge_sites << "\nleft_face_sites_active=" << (c.grains ? c.left_edge_sites : 0)
      << "\ngrain_diameter_target_grid=" << c.grain_diameter_grid << "\ngrain_diameter_target_m=" << c.grain_diameter_grid * c.dx
      << "\ngrain_count_rule=round(6*nx*ny*nz/(pi*d_grid^3)),minimum_1"
      << "\nvoronoi_sites=" << m.seeds.size() / 3 << "\nrandom_seed=" << c.random_seed
      << "\ngb_mask_FWHM_grid=" << c.gb_fwhm_grid << "\ngb_mask_FWHM_m=" << c.gb_fwhm_grid * c.dx
      << "\ngb_mask_integral_effective_width_m=" << nicr::reference_gb_width(c.gb_fwhm_grid, c.dx)
      << "\ngb_peak_mobility_factor_O=" << c.gb_factor_o << "\ngb_peak_mobility_factor_Cr=" << c.gb_factor_cr
      << "\nnucleus_shape=sphere\nnucleus_geometric_radius_grid=" << c.radius_grid
      << "\nnucleus_geometric_radius_m=" << c.radius_grid * c.dx << "\nexclusion_gap_grid=" << c.exclusion_gap_grid
      << "\nnucleation_period_s=" << c.nucleation_period << "\neta_output=" << eta_output
      << "\nmax_eta_fields=" << c.max_eta_fields << "\n";
    f << backend;
    f << "device_field_storage_MiB=" << m.device_bytes() / (1024. * 1024.)
      << "\nfield_memory_estimates=device_resident_fields_trial_buffers_and_reduction_scratch\n";
    if (m.has_eta) {
        f << "eta_fields=" << m.neta << "\neta_W=" << c.eta_W << "\neta_kappa=" << ec.K << "\neta_L=" << c.eta_L
          << "\neta_oxide_penalty=" << ec.A << "\neta_width_10_90_grid=" << 2. * std::log(9.) * ec.ell / c.dx
          << "\neta_mask_integrated_width_m=" << 8. * ec.ell / 3. << "\neta_transport_scale=" << ec.scale
          << "\neta_planar_GB_energy_model_units=" << std::sqrt(2. * ec.K * c.eta_W) / 3.
          << "\neta_planar_geometric_mobility_model_units=" << 3. * c.eta_L * ec.ell << "\n";
        if (c.eta_colours > 0)   // extension: grains coloured into eta fields
            f << "eta_init=coloured_voronoi_tanh_boundaries\neta_colours=" << c.eta_colours << "\n";
    }
    if (c.nucleation == NICR_NUC_CENTER)
        f << "initial_oxide_center_x_m=" << 0.5 * c.nx * c.dx << "\ninitial_oxide_center_y_m=" << 0.5 * c.ny * c.dy
          << "\ninitial_oxide_center_z_m=" << 0.5 * c.nz * c.dz << "\ninitial_oxide_center_i=" << 0.5 * (c.nx + 1.)
          << "\ninitial_oxide_center_j=" << 0.5 * (c.ny + 1.) << "\ninitial_oxide_center_k=" << 0.5 * (c.nz + 1.) << "\n";
    f << "mobility_note=prefactors_retained_from_uploaded_18wtpct_setup;local_M_includes_concentration_phase_and_GB_factors\n"
      << "calibration_note=eta_and_GB_transport_parameters_require_material_calibration\n";
    std::ofstream g(out + "/grains.csv");
    g << "grain_id,seed_x_grid,seed_y_grid,seed_z_grid,volume_cells,volume_m3,equivalent_diameter_grid,equivalent_diameter_m\n";
    long double mean = 0.;
    for (size_t q = 0; q < m.volumes.size(); ++q) {
        const double d = std::cbrt(6. * m.volumes[q] / pi);
        mean += d;
        g << std::setprecision(17) << q + 1 << "," << m.seeds[3 * q] << "," << m.seeds[3 * q + 1] << "," << m.seeds[3 * q + 2]
          << "," << m.volumes[q] << "," << m.volumes[q] * c.dx * c.dy * c.dz << "," << d << "," << d * c.dx << "\n";
    }
    mean /= m.volumes.size();
    f << "measured_arithmetic_mean_equivalent_diameter_grid=" << mean << "\n";
    if (!f || !g) throw nicr::Error(NICR_ERR_IO, "Metadata write failed.");
}

template <class Fn>
int guarded(nicr_handle* h, Fn fn) {
    if (!h || !h->m) return NICR_ERR_INVALID_ARG;
    try {
        fn(*h->m);
        return NICR_OK;
    } catch (const nicr::Error& e) {
        h->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        h->err = e.what();
        return NICR_ERR_IO;
    }
}

void copy_out(char* buf, size_t len, const std::string& s) {
    if (!buf || !len) return;
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = 0;
}

int self_test(int dim) { return nicr::run_self_test(dim); }

// ------------------------------------------------------------------ run()
// The program over a slab group (--slabs N [--slab-devices a,b,...]): the
// domain split along X over N slabs, slab i on GPU a_i (default: GPU i modulo
// the GPUs present). The same files as the single-GPU program: diagnostics,
// grain statistics and VTI frames are whole-domain values gathered from the
// slabs; parameters.txt names the slab backend and the summed device memory.
// Checkpoints and ASCII VTK frames are not written in this form.
int run_program_slabs(const nicr_config& c, int dim, const std::string& dir, int slabs, const std::string& devs,
                      const std::string& restart) {
    try {
        if (dim != 3) throw std::runtime_error("--slabs needs the 3D program.");
        if (!restart.empty() || c.checkpoint_every > 0)
            throw std::runtime_error("--slabs does not write or read checkpoints.");
        if (!c.output_vti) throw std::runtime_error("--slabs writes VTI frames only (--output-format vti).");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw std::runtime_error("no CUDA device is available");
        std::vector<int> dev;
        if (!devs.empty()) {
            std::stringstream ss(devs);
            std::string item;
            while (std::getline(ss, item, ',')) dev.push_back(std::stoi(item));
            if (slabs == 1) slabs = (int)dev.size();
            if ((int)dev.size() != slabs) throw std::runtime_error("--slab-devices needs one device per slab.");
        } else {
            for (int s = 0; s < slabs; ++s) dev.push_back((c.device + s) % count);
        }
        if (fs::exists(dir) && !fs::is_empty(dir)) throw std::runtime_error("Output directory is not empty; choose a new --out.");
        fs::create_directories(dir);
        nicr::SlabGroup g(c, slabs, dev.data());
        const bool has_eta = g.m[0]->has_eta;
        const int neta = g.m[0]->neta;
        metadata(meta_of(g), dir);
        std::ofstream log(dir + "/diagnostics.csv"), gd, gh;
        if (!log) throw std::runtime_error("Cannot open diagnostics.csv");
        log << "step,time_s,sum_O,sum_Cr,mean_phi,O_boundary,O_seed,Cr_seed,O_Ck,Cr_Ck,O_clipping,Cr_clipping,"
               "O_budget_residual,Cr_budget_residual,nuclei,clipped_cells,min_O,max_O,min_Cr,max_Cr,min_Ni,min_phi,max_phi"
               ",mean_h_phi,oxide_volume_m3\n";
        if (has_eta) {
            gd.open(dir + "/grain_diagnostics.csv");
            gh.open(dir + "/grain_history.csv");
            if (!gd || !gh) throw std::runtime_error("Cannot open grain diagnostics.");
            gd << "step,time_s,min_eta,max_eta,min_sum_eta2,max_sum_eta2,mean_sum_eta2,grains_with_metal_cells,"
                  "unassigned_metal_cells,integrated_active_GB_m3,max_GB_mask,grain_energy_model_units\n";
            gh << "step,time_s,grain_id,dominant_metal_cells,weighted_metal_volume_cells,weighted_metal_volume_m3\n";
        }
        auto do_log = [&](int n) {
            nicr_diagnostics d;
            g.diagnostics(&d);
            nicr_budget b;
            g.budget(&b);
            log << log_row(c, dim, d, b, n);
            if (has_eta) {
                nicr_grain_stats st;
                std::vector<long long> cells((size_t)neta);
                std::vector<double> amount((size_t)neta * 2);
                g.grain_stats(&st, cells.data(), amount.data());
                std::string a, bb;
                grain_rows(c, dim, neta, st, cells, amount, n, a, bb);
                gd << a;
                gh << bb;
            }
        };
        auto frame = [&](const std::string& path) {
            std::vector<unsigned char> arrays;
            const bool f64 = c.output_float64 != 0;
            const unsigned r = g.vti_arrays(arrays, f64);
            if (r) {
                int arr = 0;
                while (!(r & (1u << arr))) ++arr;
                throw nicr::Error(NICR_ERR_IO, std::string("VTI ") + NAMES3[(size_t)arr] +
                                                   " exceeds output type range; use --output-precision float64.");
            }
            compose_vti(c, arrays.data(), f64, path);
        };
        do_log(0);
        frame(dir + "/fields_0.vti");
        std::cout << "EXECUTION BACKEND: CUDA sm_100a, the domain split along X over " << slabs << " slabs.\n";
        std::cout << "MPI processes: 1 (slabs on GPUs";
        for (int d : dev) std::cout << " " << d;
        std::cout << ")\n";
        std::cout << "Output: vti, " << (c.output_float64 ? "float64" : "float32") << "; zlib level=" << c.compression_level
                  << "; frozen-eta cache=" << (c.frozen_eta_cache ? "on" : "off") << ".\n";
        std::cout << "Version " << VERSION3 << "; grains=" << (c.grains ? "on" : "off")
                  << "; oxygen_diffusion=" << (c.oxygen_diffusion ? "on" : "off") << "; nucleation="
                  << (c.nucleation == NICR_NUC_CENTER ? "center" : c.nucleation == NICR_NUC_OFF ? "off" : "ksp") << "; "
                  << g.m[0]->seeds.size() / 3 << " grain(s).\n";
        int last = 0, n = 0;
        try {
            while (n < c.steps) {
                int next = std::min(c.steps, (n / 1000 + 1) * 1000);
                next = std::min(next, (n / c.output_every + 1) * c.output_every);
                int done = 0;
                const int r = g.advance(next - n, true, &done);
                last = n + done;
                if (r != NICR_OK) throw nicr::Error(r, g.err);
                n = next;
                if (n % 1000 == 0 || n == c.steps)
                    std::cout << "step " << n << "/" << c.steps << " (" << 100.0 * n / c.steps << "%), time=" << n * c.dt
                              << " s" << std::endl;
                if (n % c.output_every == 0 || n == c.steps) {
                    do_log(n);
                    log.flush();
                    if (!log) throw std::runtime_error("Diagnostics write failed.");
                    if (has_eta) {
                        gd.flush();
                        gh.flush();
                        if (!gd || !gh) throw std::runtime_error("Grain diagnostics write failed.");
                    }
                    frame(dir + "/fields_" + std::to_string(n) + ".vti");
                }
            }
        } catch (const std::exception& e) {
            std::ofstream stop(dir + "/STOPPED.txt");
            stop << "Last accepted time step: " << last << "\n" << e.what() << "\n";
            frame(dir + "/state_at_failure.vti");
            throw;
        }
        std::cout << "Finished " << last << " steps. Output: " << dir << "\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << "\n";
        return 1;
    }
}

int run_program(int dim, int argc, const char* const* argv) {
    nicr_config c;
    std::vector<char> out(4096), err(16384);
    int self = 0;
    // --restart FILE is a program-level flag (the state to continue from); the
    // rest is the configuration
    std::string restart, slab_devices;
    int slabs = 1;
    std::vector<const char*> args;
    for (int q = 0; q < argc; ++q) {
        const std::string a = q > 0 ? argv[q] : "";
        if (a == "--restart" || a == "--slabs" || a == "--slab-devices") {
            if (q + 1 >= argc) {
                std::cerr << "ERROR: Missing value for " << a << "\n";
                return 1;
            }
            const std::string v = argv[++q];
            if (a == "--restart") restart = v;
            else if (a == "--slab-devices") slab_devices = v;
            else {
                size_t used = 0;
                try { slabs = std::stoi(v, &used); } catch (...) { used = 0; }
                if (used != v.size() || slabs < 1 || slabs > nicr::kMaxSlabs) {
                    std::cerr << "ERROR: --slabs expects an integer in [1, 16].\n";
                    return 1;
                }
            }
            continue;
        }
        args.push_back(argv[q]);
    }
    argc = (int)args.size();
    argv = args.data();
    const int rc = nicr_config_parse(&c, dim, argc - 1, argv + 1, out.data(), out.size(), &self, err.data(), err.size());
    if (rc == 100) {
        std::cout << err.data();
        return 0;
    }
    if (rc != NICR_OK) {
        std::cerr << "ERROR: " << err.data() << "\n";
        return 1;
    }
    if (self) return self_test(dim);
    const std::string dir = out.data();
    if (slabs > 1 || !slab_devices.empty()) return run_program_slabs(c, dim, dir, slabs, slab_devices, restart);
    try {
        if (fs::exists(dir) && !fs::is_empty(dir)) throw std::runtime_error("Output directory is not empty; choose a new --out.");
        fs::create_directories(dir);
        Model m(c);
        if (!restart.empty()) m.load_state(restart);
        const int start = (int)m.steps_done;
        metadata(meta_of(m), dir);
        std::ofstream log(dir + "/diagnostics.csv"), gd, gh;
        if (!log) throw std::runtime_error("Cannot open diagnostics.csv");
        log << "step,time_s,sum_O,sum_Cr,mean_phi,O_boundary,O_seed,Cr_seed,O_Ck,Cr_Ck,O_clipping,Cr_clipping,"
               "O_budget_residual,Cr_budget_residual,nuclei,clipped_cells,min_O,max_O,min_Cr,max_Cr,min_Ni,min_phi,max_phi"
            << (dim == 3 ? ",mean_h_phi,oxide_volume_m3" : "") << "\n";
        if (m.has_eta) {
            gd.open(dir + "/grain_diagnostics.csv");
            gh.open(dir + "/grain_history.csv");
            if (!gd || !gh) throw std::runtime_error("Cannot open grain diagnostics.");
            gd << "step,time_s,min_eta,max_eta,min_sum_eta2,max_sum_eta2,mean_sum_eta2,grains_with_metal_cells,"
                  "unassigned_metal_cells,"
               << (dim == 3 ? "integrated_active_GB_m3,max_GB_mask,grain_energy_model_units\n"
                            : "integrated_active_GB_m2,max_GB_mask,grain_energy_per_depth\n");
            gh << "step,time_s,grain_id,dominant_metal_cells,"
               << (dim == 3 ? "weighted_metal_volume_cells,weighted_metal_volume_m3\n"
                            : "weighted_metal_area_cells,weighted_metal_area_m2\n");
        }
        auto do_log = [&](int n) {
            log << log_row(m, n);
            if (m.has_eta) {
                std::string a, b;
                grain_rows(m, n, a, b);
                gd << a;
                gh << b;
            }
        };
        auto checkpoint = [&](int n) {
            if (c.checkpoint_every <= 0 || n % c.checkpoint_every != 0) return;
            m.save_state(dir + "/checkpoint.bin.tmp");
            fs::rename(dir + "/checkpoint.bin.tmp", dir + "/checkpoint.bin");
        };
        do_log(start);
        write_visualization(m, dir + "/fields_" + std::to_string(start));
        std::cout << "EXECUTION BACKEND: CUDA sm_100a, one GPU holds the whole domain.\n";
        std::cout << "MPI processes: 1 (domain resident on one GPU)\n";
        if (dim == 3)
            std::cout << "Output: " << (c.output_vti ? "vti" : "vtk") << ", "
                      << (!c.output_vti ? "ASCII Float64" : (c.output_float64 ? "float64" : "float32"))
                      << "; zlib level=" << c.compression_level
                      << "; frozen-eta cache=" << (c.frozen_eta_cache ? "on" : "off") << ".\n";
        std::cout << "Version " << (dim == 3 ? VERSION3 : VERSION2) << "; grains=" << (c.grains ? "on" : "off")
                  << "; oxygen_diffusion=" << (c.oxygen_diffusion ? "on" : "off") << "; nucleation="
                  << (c.nucleation == NICR_NUC_CENTER ? "center" : c.nucleation == NICR_NUC_OFF ? "off" : "ksp") << "; "
                  << m.seeds.size() / dim << " grain(s).\n";
        int last = start, n = start;
        try {
            while (n < c.steps) {
                // advance to the next progress line, output or checkpoint, in one batch
                int next = std::min(c.steps, (n / 1000 + 1) * 1000);
                next = std::min(next, (n / c.output_every + 1) * c.output_every);
                if (c.checkpoint_every > 0) next = std::min(next, (n / c.checkpoint_every + 1) * c.checkpoint_every);
                int done = 0;
                const int r = m.run(next - n, &done);
                last = n + done;
                if (r != NICR_OK) throw nicr::Error(r, m.last_error);
                n = next;
                if (n % 1000 == 0 || n == c.steps)
                    std::cout << "step " << n << "/" << c.steps << " (" << 100.0 * n / c.steps << "%), time=" << n * c.dt
                              << " s" << std::endl;
                if (n % c.output_every == 0 || n == c.steps) {
                    do_log(n);
                    log.flush();
                    if (!log) throw std::runtime_error("Diagnostics write failed.");
                    if (m.has_eta) {
                        gd.flush();
                        gh.flush();
                        if (!gd || !gh) throw std::runtime_error("Grain diagnostics write failed.");
                    }
                    write_visualization(m, dir + "/fields_" + std::to_string(n), true);
                }
                checkpoint(n);
            }
            output_wait(m);
        } catch (const std::exception& e) {
            try {
                output_wait(m);   // the failure is reported; a pending frame is completed if it can be
            } catch (const std::exception&) {
            }
            std::ofstream stop(dir + "/STOPPED.txt");
            stop << "Last accepted time step: " << last << "\n" << e.what() << "\n";
            write_visualization(m, dir + "/state_at_failure");
            throw;
        }
        std::cout << "Finished " << last << " steps. Output: " << dir << "\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << "\n";
        return 1;
    }
}

}  // namespace

// ------------------------------------------------------------------ C-ABI
extern "C" {

int nicr_slabs_write_vti(nicr_slabs* s, const char* path) {
    nicr::SlabGroup* g = nicr_slabs_group(s);
    if (!g || !path) return NICR_ERR_INVALID_ARG;
    try {
        std::vector<unsigned char> arrays;
        const bool f64 = g->c.output_float64 != 0;
        const unsigned r = g->vti_arrays(arrays, f64);
        if (r) {
            int arr = 0;
            while (!(r & (1u << arr))) ++arr;
            throw nicr::Error(NICR_ERR_IO, std::string("VTI ") + NAMES3[(size_t)arr] +
                                               " exceeds output type range; use --output-precision float64.");
        }
        compose_vti(g->c, arrays.data(), f64, path);
        return NICR_OK;
    } catch (const nicr::Error& e) {
        nicr_slabs_set_error(s, e.what());
        return e.code;
    } catch (const std::exception& e) {
        nicr_slabs_set_error(s, e.what());
        return NICR_ERR_IO;
    }
}

int nicr_write_vtk(nicr_handle* h, const char* path) {
    return guarded(h, [&](Model& m) {
        if (m.dim == 2) write_vtk2(m, path);
        else write_vtk3(m, path);
    });
}
int nicr_write_vti(nicr_handle* h, const char* path) {
    return guarded(h, [&](Model& m) {
        if (m.dim != 3) throw nicr::Error(NICR_ERR_STATE, "VTI output exists only in 3D");
        write_vti3(m, path);
    });
}
int nicr_write_vti_async(nicr_handle* h, const char* path) {
    return guarded(h, [&](Model& m) {
        if (m.dim != 3) throw nicr::Error(NICR_ERR_STATE, "VTI output exists only in 3D");
        write_vti3_async(m, path);
    });
}
int nicr_output_wait(nicr_handle* h) {
    return guarded(h, [&](Model& m) { output_wait(m); });
}
int nicr_write_metadata(nicr_handle* h, const char* out_dir) {
    return guarded(h, [&](Model& m) { metadata(meta_of(m), out_dir); });
}
int nicr_format_log_row(nicr_handle* h, int n, char* buf, size_t len) {
    return guarded(h, [&](Model& m) { copy_out(buf, len, log_row(m, n)); });
}
int nicr_format_grain_rows(nicr_handle* h, int n, char* diag, size_t diag_len, char* history, size_t history_len) {
    return guarded(h, [&](Model& m) {
        std::string a, b;
        grain_rows(m, n, a, b);
        copy_out(diag, diag_len, a);
        copy_out(history, history_len, b);
    });
}
int nicr_main(int dim, int argc, const char* const* argv) {
    if (dim != 2 && dim != 3) return 1;
    return run_program(dim, argc, argv);
}

}  // extern "C"
