// sifv_vtk.cpp -- VTK XML output of one rank's interior cells, file for file
// and byte for byte what VTKSession / VTKWriter write (src/VTKSession.cpp,
// src/VTKWriter.cpp): ASCII RectilinearGrid pieces (.vtr), their parallel
// meta-files (.pvtr) and the .pvd time series.
//
// The reference formats doubles through an ostream at precision 15, which
// is printf's %.15g; std::to_chars(general, 15) is specified as the same
// conversion and runs an order of magnitude faster.  Rows of a data array
// are formatted by several threads into separate buffers and written in
// order, so the bytes do not depend on the thread count.  A session owns one
// writer thread: writes queued from the device path (sifv_vtk_write) are
// formatted while the solver keeps stepping.
#include <algorithm>
#include <charconv>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "sifv.h"
#include "sifv_vtk_api.h"

struct sifv_vtk {
    std::string dir, base;
    sifv::VtkLayout L{};
    std::vector<double> xn, yn, zn;   // node coordinates (nx+1, ny+1, nz+1)
    int nThreads = 1;
    int fileNum = 0;
    // writer thread
    std::mutex mu;
    std::condition_variable cv, idle;
    std::deque<std::function<int(std::string&)>> jobs;
    bool stop = false, busy = false;
    int firstErr = SIFV_OK;
    std::string err;
    std::thread worker;
    void* stage = nullptr;
    void (*releaseStage)(void*) = nullptr;
};

namespace sifv {
namespace {

thread_local std::string g_vtkErr;

const std::string kPvdFooter = "  </Collection>\n</VTKFile>\n";

void put(std::string& s, double v) {
    char buf[40];
    auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 15);
    s.append(buf, r.ptr);
}

bool ensure_parent(const std::string& path, std::string& err) {
    std::error_code ec;
    auto parent = std::filesystem::path(path).parent_path();
    if (!parent.empty()) std::filesystem::create_directories(parent, ec);
    if (ec) {
        err = "cannot create directory " + parent.string() + ": " + ec.message();
        return false;
    }
    return true;
}

// The rows (j, k) of one data array, formatted in parallel: each row is
// "         " + the text of its cells + "\n".
template <typename CellFn>
void format_rows(const sifv_vtk* v, std::string& out, CellFn cell) {
    const VtkLayout& L = v->L;
    const long long rows = (long long)L.ny * L.nz;
    const long long cells = rows * L.nx;
    int T = (cells < 65536) ? 1 : std::max(1, std::min<int>(v->nThreads, (int)std::min<long long>(rows, 256)));
    std::vector<std::string> part(T);
    auto work = [&](int t) {
        std::string& s = part[t];
        long long r0 = rows * t / T, r1 = rows * (t + 1) / T;
        s.reserve((size_t)((r1 - r0) * ((long long)L.nx * 24 + 10)));
        for (long long r = r0; r < r1; ++r) {
            int j = (int)(r % L.ny), k = (int)(r / L.ny);
            s += "         ";
            for (int i = 0; i < L.nx; ++i) cell(s, i, j, k);
            s += '\n';
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 1; t < T; ++t) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
    }
    for (auto& p : part) out += p;
}

size_t gidx(const VtkLayout& L, int i, int j, int k) {
    const size_t nxT = (size_t)L.nx + 2 * L.ngx, nyT = (size_t)L.ny + 2 * L.ngy;
    return (size_t)(i + L.ngx) + nxT * ((size_t)(j + L.ngy) + nyT * (size_t)(k + L.ngz));
}

bool write_file(const std::string& file, const std::string& s, const char* who, std::string& err) {
    if (!ensure_parent(file, err)) return false;
    std::ofstream o(file, std::ios::binary);
    if (!o.is_open()) {
        err = std::string(who) + ": cannot open " + file;
        return false;
    }
    o.write(s.data(), (std::streamsize)s.size());
    if (!o) err = std::string(who) + ": write failed on " + file;
    return (bool)o;
}

// VTKWriter::writeVTR (src/VTKWriter.cpp:20-190) for the single piece with
// extent {0, nx, 0, ny, 0, nz} and the "Rank" array of rank 0.
bool write_vtr(const sifv_vtk* v, const std::string& file, const sifv_vtk_fields_t* f, std::string& err) {
    const VtkLayout& L = v->L;
    std::string s;
    s.reserve(1 << 16);
    const std::string ext =
        "0 " + std::to_string(L.nx) + " 0 " + std::to_string(L.ny) + " 0 " + std::to_string(L.nz);
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"RectilinearGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    s += "  <RectilinearGrid WholeExtent=\"" + ext + "\">\n";
    s += "    <Piece Extent=\"" + ext + "\">\n";
    s += "      <Coordinates>\n";
    s += "        <DataArray type=\"Float64\" Name=\"X\" format=\"ascii\">\n";
    s += "         ";
    for (int i = 0; i <= L.nx; ++i) {
        s += ' ';
        put(s, v->xn[i]);
    }
    s += "\n        </DataArray>\n";
    const double dx0 = v->xn[1] - v->xn[0], dy0 = v->yn[1] - v->yn[0];
    s += "        <DataArray type=\"Float64\" Name=\"Y\" format=\"ascii\">\n";
    s += "         ";
    if (L.ny == 1) {   // one cell in y: a slab 0 .. first x width
        s += " 0.0 ";
        put(s, dx0);
    } else {
        for (int j = 0; j <= L.ny; ++j) {
            s += ' ';
            put(s, v->yn[j]);
        }
    }
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"Float64\" Name=\"Z\" format=\"ascii\">\n";
    s += "         ";
    if (L.nz == 1) {   // one cell in z: a slab 0 .. min(dx0, dy0, 1)
        s += " 0.0 ";
        put(s, std::min(dx0, std::min(dy0, 1.0)));
    } else {
        for (int k = 0; k <= L.nz; ++k) {
            s += ' ';
            put(s, v->zn[k]);
        }
    }
    s += "\n        </DataArray>\n";
    s += "      </Coordinates>\n";
    s += "      <CellData>\n";

    auto scalar = [&](const std::string& name, const double* a) -> bool {
        if (!a) {
            err = "VTK field " + name + " missing";
            return false;
        }
        s += "        <DataArray type=\"Float64\" Name=\"" + name + "\" format=\"ascii\">\n";
        format_rows(v, s, [&](std::string& o, int i, int j, int k) {
            o += ' ';
            put(o, a[gidx(L, i, j, k)]);
        });
        s += "        </DataArray>\n";
        return true;
    };
    auto vector = [&](const std::string& name, const double* const* a) -> bool {
        for (int d = 0; d < L.dim; ++d)
            if (!a[d]) {
                err = "VTK field " + name + " missing";
                return false;
            }
        s += "        <DataArray type=\"Float64\" Name=\"" + name + "\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        format_rows(v, s, [&](std::string& o, int i, int j, int k) {
            const size_t c = gidx(L, i, j, k);
            o += ' ';
            put(o, a[0][c]);
            o += ' ';
            put(o, L.dim >= 2 ? a[1][c] : 0.0);
            o += ' ';
            put(o, L.dim >= 3 ? a[2][c] : 0.0);
        });
        s += "        </DataArray>\n";
        return true;
    };
    if (!scalar("Pressure", f->pres)) return false;
    if (L.useIGR && !scalar("Sigma", f->sigma)) return false;
    if (!scalar("TotalEnergy", f->rhoE)) return false;
    if (!vector("Velocity", f->vel) || !vector("Momentum", f->mom)) return false;
    if (L.nPhases <= 0 && !scalar("Density", f->rho)) return false;
    for (int p = 0; p < L.nPhases; ++p)
        if (!scalar("AlphaRho_" + std::to_string(p), f->alphaRho[p])) return false;
    for (int p = 0; p < L.nPhases; ++p)
        if (!scalar("Alpha_" + std::to_string(p), f->alpha[p])) return false;
    s += "        <DataArray type=\"Int32\" Name=\"Rank\" format=\"ascii\">\n";
    format_rows(v, s, [](std::string& o, int, int, int) { o += " 0"; });
    s += "        </DataArray>\n";
    s += "      </CellData>\n";
    s += "    </Piece>\n";
    s += "  </RectilinearGrid>\n";
    s += "</VTKFile>\n";
    return write_file(file, s, "VTKWriter::writeVTR", err);
}

// VTKWriter::writePVTR (src/VTKWriter.cpp:192-246) for one piece.
bool write_pvtr(const sifv_vtk* v, const std::string& file, const std::string& piece, std::string& err) {
    const VtkLayout& L = v->L;
    std::string s;
    const std::string ext =
        "0 " + std::to_string(L.nx) + " 0 " + std::to_string(L.ny) + " 0 " + std::to_string(L.nz);
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"PRectilinearGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    s += "  <PRectilinearGrid WholeExtent=\"" + ext + "\" GhostLevel=\"0\">\n";
    s += "    <PCoordinates>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"X\"/>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"Y\"/>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"Z\"/>\n";
    s += "    </PCoordinates>\n";
    s += "    <PCellData>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"Pressure\"/>\n";
    if (L.useIGR) s += "      <PDataArray type=\"Float64\" Name=\"Sigma\"/>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"TotalEnergy\"/>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"Velocity\" NumberOfComponents=\"3\"/>\n";
    s += "      <PDataArray type=\"Float64\" Name=\"Momentum\" NumberOfComponents=\"3\"/>\n";
    if (L.nPhases <= 0) s += "      <PDataArray type=\"Float64\" Name=\"Density\"/>\n";
    for (int p = 0; p < L.nPhases; ++p)
        s += "      <PDataArray type=\"Float64\" Name=\"AlphaRho_" + std::to_string(p) + "\"/>\n";
    for (int p = 0; p < L.nPhases; ++p)
        s += "      <PDataArray type=\"Float64\" Name=\"Alpha_" + std::to_string(p) + "\"/>\n";
    s += "      <PDataArray type=\"Int32\" Name=\"Rank\"/>\n";
    s += "    </PCellData>\n";
    s += "    <Piece Extent=\"" + ext + "\" Source=\"" + piece + "\"/>\n";
    s += "  </PRectilinearGrid>\n";
    s += "</VTKFile>\n";
    return write_file(file, s, "VTKWriter::writePVTR", err);
}

// VTKWriter::writePVD (src/VTKWriter.cpp:248-291): create = header +
// footer; otherwise the footer is replaced by one DataSet line + footer.
bool write_pvd(const std::string& file, bool create, double time, const std::string& data, std::string& err) {
    if (create) {
        std::string s = "<?xml version=\"1.0\"?>\n";
        s += "<VTKFile type=\"Collection\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
        s += "  <Collection>\n";
        s += kPvdFooter;
        return write_file(file, s, "VTKWriter::writePVD", err);
    }
    std::error_code ec;
    auto size = std::filesystem::file_size(file, ec);
    if (ec || size < kPvdFooter.size()) {
        err = "VTKWriter::writePVD: cannot open " + file;
        return false;
    }
    std::filesystem::resize_file(file, size - kPvdFooter.size(), ec);
    std::ofstream o(file, std::ios::binary | std::ios::app);
    if (ec || !o.is_open()) {
        err = "VTKWriter::writePVD: cannot open " + file;
        return false;
    }
    std::string s = "    <DataSet timestep=\"";
    put(s, time);
    s += "\" file=\"" + data + "\"/>\n";
    s += kPvdFooter;
    o.write(s.data(), (std::streamsize)s.size());
    return (bool)o;
}

void writer_main(sifv_vtk* v) {
    for (;;) {
        std::function<int(std::string&)> job;
        {
            std::unique_lock<std::mutex> lk(v->mu);
            v->cv.wait(lk, [&] { return v->stop || !v->jobs.empty(); });
            if (v->jobs.empty()) return;
            job = std::move(v->jobs.front());
            v->jobs.pop_front();
            v->busy = true;
        }
        std::string e;
        int st = job(e);
        {
            std::lock_guard<std::mutex> lk(v->mu);
            if (st != SIFV_OK && v->firstErr == SIFV_OK) {
                v->firstErr = st;
                v->err = e;
            }
            v->busy = false;
        }
        v->idle.notify_all();
    }
}

}  // namespace

int vtk_next_file(sifv_vtk_t* v) { return v->fileNum++; }

void vtk_enqueue(sifv_vtk_t* v, std::function<int(std::string&)> job) {
    {
        std::lock_guard<std::mutex> lk(v->mu);
        v->jobs.push_back(std::move(job));
    }
    v->cv.notify_one();
}

const VtkLayout& vtk_layout(const sifv_vtk_t* v) { return v->L; }

void vtk_set_stage(sifv_vtk_t* v, void* stage, void (*release)(void*)) {
    v->stage = stage;
    v->releaseStage = release;
}

void* vtk_stage(sifv_vtk_t* v) { return v->stage; }

// VTKSession::write (src/VTKSession.cpp:24-60) for rank 0 of 1.
int vtk_write_snapshot(sifv_vtk_t* v, int n, double time, const sifv_vtk_fields_t* f, std::string& err) {
    const std::string snap = "snapshot_" + std::to_string(n);
    const std::string vtr = v->base + "_" + std::to_string(n) + "_r0.vtr";
    const std::string pvtr = v->base + "_" + std::to_string(n) + ".pvtr";
    if (!write_vtr(v, v->dir + "/" + snap + "/" + vtr, f, err)) return SIFV_ERR_BAD_ARG;
    if (!write_pvtr(v, v->dir + "/" + snap + "/" + pvtr, vtr, err)) return SIFV_ERR_BAD_ARG;
    if (!write_pvd(v->dir + "/" + v->base + ".pvd", false, time, snap + "/" + pvtr, err)) return SIFV_ERR_BAD_ARG;
    return SIFV_OK;
}

}  // namespace sifv

using namespace sifv;

extern "C" {

int sifv_vtk_open(const char* dir, const char* baseName, const sifv_config_t* cfg, const sifv_mesh_t* mesh,
                  int nThreads, sifv_vtk_t** out) {
    if (!out) {
        g_vtkErr = "null argument";
        return SIFV_ERR_BAD_ARG;
    }
    *out = nullptr;
    if (!dir || !baseName || !cfg || !mesh || !mesh->xNodes) {
        g_vtkErr = "null argument";
        return SIFV_ERR_BAD_ARG;
    }
    const int dim = cfg->dim;
    if (dim < 1 || dim > 3 || mesh->nx < 1 || (dim >= 2 && (mesh->ny < 1 || !mesh->yNodes)) ||
        (dim >= 3 && (mesh->nz < 1 || !mesh->zNodes)) || cfg->nPhases < 0 || cfg->nPhases > SIFV_MAX_PHASES ||
        cfg->nGhost < 0) {
        g_vtkErr = "bad mesh or configuration";
        return SIFV_ERR_BAD_ARG;
    }
    auto* v = new sifv_vtk();
    v->dir = dir;
    v->base = baseName;
    VtkLayout& L = v->L;
    L.dim = dim;
    L.nx = mesh->nx;
    L.ny = dim >= 2 ? mesh->ny : 1;
    L.nz = dim >= 3 ? mesh->nz : 1;
    L.ngx = cfg->nGhost;
    L.ngy = dim >= 2 ? cfg->nGhost : 0;
    L.ngz = dim >= 3 ? cfg->nGhost : 0;
    L.nPhases = cfg->nPhases;
    L.useIGR = cfg->useIGR ? 1 : 0;
    v->xn.assign(mesh->xNodes, mesh->xNodes + L.nx + 1);
    if (dim >= 2) v->yn.assign(mesh->yNodes, mesh->yNodes + L.ny + 1);
    else v->yn = {0.0, 1.0};
    if (dim >= 3) v->zn.assign(mesh->zNodes, mesh->zNodes + L.nz + 1);
    else v->zn = {0.0, 1.0};
    if (nThreads <= 0) nThreads = (int)std::max(1u, std::thread::hardware_concurrency());
    v->nThreads = nThreads;
    std::string err;
    if (!write_pvd(v->dir + "/" + v->base + ".pvd", true, 0.0, "", err)) {
        g_vtkErr = err;
        delete v;
        return SIFV_ERR_BAD_ARG;
    }
    v->worker = std::thread(writer_main, v);
    *out = v;
    return SIFV_OK;
}

int sifv_vtk_write_host(sifv_vtk_t* v, double time, const sifv_vtk_fields_t* f) {
    if (!v || !f) return SIFV_ERR_BAD_ARG;
    const int n = vtk_next_file(v);
    const sifv_vtk_fields_t copy = *f;
    vtk_enqueue(v, [v, n, time, copy](std::string& e) { return vtk_write_snapshot(v, n, time, &copy, e); });
    return sifv_vtk_flush(v);
}

int sifv_vtk_flush(sifv_vtk_t* v) {
    if (!v) return SIFV_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(v->mu);
    v->idle.wait(lk, [&] { return v->jobs.empty() && !v->busy; });
    return v->firstErr;
}

int sifv_vtk_close(sifv_vtk_t* v) {
    if (!v) return SIFV_ERR_BAD_ARG;
    int st = sifv_vtk_flush(v);
    {
        std::lock_guard<std::mutex> lk(v->mu);
        v->stop = true;
    }
    v->cv.notify_all();
    if (v->worker.joinable()) v->worker.join();
    if (v->releaseStage) v->releaseStage(v->stage);
    delete v;
    return st;
}

const char* sifv_vtk_last_error(const sifv_vtk_t* v) {
    if (!v) return g_vtkErr.c_str();
    return v->err.c_str();
}

}  // extern "C"
