// fdtd_io.cpp — the reference's output files of a solve.
//
//   binary matrix    IO::writeMatrixX<double>(..., IO::BINARY) (utils/IO/IO.h:107-160)
//                    and MATRIX::write (linearalgebra/MATRIX_FAST.cpp:134-155): int32
//                    rows, int32 cols, then rows*cols doubles, row-major
//   snapshot         FDTD_AcousticSimulator::_SaveSimulationSnapshot
//                    (FDTD_AcousticSimulator.cpp:381-415, USE_COLLOCATED) with the
//                    data of PML_WaveSolver::GetAllSimulationData (PML_WaveSolver.cpp:510-520)
//   solver config    SaveSolverConfig's position files (FDTD_AcousticSimulator.cpp:146-230, :647-661)
//   field dumps      _SavePressureTimestep / _SaveVelocityTimestep (:253-307): x fastest
//
// File names are composed as CompositeFilename does (FDTD_AcousticSimulator.cpp:109-125):
// the output pattern's "%s" replaced by the file name.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

using namespace fdtd;

namespace {

bool compose(const char* pattern, const std::string& name, std::string& out) {
    const std::string pat = (pattern && *pattern) ? pattern : "%s";
    const size_t k = pat.find("%s");
    if (k == std::string::npos) return false;
    out = pat.substr(0, k) + name + pat.substr(k + 2);
    return true;
}

fdtd_status write_matrix(const std::string& path, int rows, int cols, const double* data) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return (set_error(nullptr, "cannot open " + path), FDTD_ERR_IO);
    const int32_t r = rows, c = cols;
    bool ok = std::fwrite(&r, sizeof(r), 1, f) == 1 && std::fwrite(&c, sizeof(c), 1, f) == 1;
    const size_t n = (size_t)rows * (size_t)cols;
    if (ok && n) ok = std::fwrite(data, sizeof(double), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return (set_error(nullptr, "short write to " + path), FDTD_ERR_IO);
    return FDTD_OK;
}

// full-state fields only: the reduced PML state has no split pressures or velocities to save
fdtd_status need_full_state(fdtd_solver* s) {
    if (s->region.red)
        return (set_error(s, "this FP32 solve keeps the reduced PML state; create it with pml_state = "
                             "FDTD_PML_STATE_FULL to save or load snapshots"),
                FDTD_ERR_UNSUPPORTED);
    return FDTD_OK;
}

}  // namespace

extern "C" {

fdtd_status fdtd_matrix_write(const char* path, int32_t rows, int32_t cols, const double* data) {
    if (!path || rows < 0 || cols < 0 || (!data && (int64_t)rows * cols > 0))
        return (set_error(nullptr, "fdtd_matrix_write: invalid arguments"), FDTD_ERR_INVALID_ARG);
    return write_matrix(path, rows, cols, data);
}

fdtd_status fdtd_matrix_read(const char* path, int32_t* rows, int32_t* cols, double* data, int64_t capacity) {
    if (!path || !rows || !cols) return (set_error(nullptr, "fdtd_matrix_read: invalid arguments"), FDTD_ERR_INVALID_ARG);
    FILE* f = std::fopen(path, "rb");
    if (!f) return (set_error(nullptr, std::string("cannot open ") + path), FDTD_ERR_IO);
    int32_t r = 0, c = 0;
    if (std::fread(&r, sizeof(r), 1, f) != 1 || std::fread(&c, sizeof(c), 1, f) != 1 || r < 0 || c < 0) {
        std::fclose(f);
        return (set_error(nullptr, std::string("not a binary matrix file: ") + path), FDTD_ERR_IO);
    }
    *rows = r;
    *cols = c;
    const int64_t n = (int64_t)r * c;
    fdtd_status st = FDTD_OK;
    if (data) {
        if (capacity < n) st = (set_error(nullptr, "fdtd_matrix_read: buffer smaller than rows*cols"), FDTD_ERR_INVALID_ARG);
        else if (n > 0 && std::fread(data, sizeof(double), (size_t)n, f) != (size_t)n)
            st = (set_error(nullptr, std::string("short read from ") + path), FDTD_ERR_IO);
    }
    std::fclose(f);
    return st;
}

// _SaveSimulationSnapshot(numbering): p_pml_<d>, v_pml_<d>, p_collocated_<d> (d = 0..2),
// p_pml_full and the ASCII p_collocated_ind.  After n steps the reference's current
// collocated buffer is (1 + n) % 3 (Reinitialize_PML_WaveSolver sets 1, each step
// advances it); its previous one is (ind + 2) % 3.  The third buffer only holds a
// value the next step overwrites before reading it; it is written as zeros.
// _pFull is never stepped on the collocated path: zeros, as in the reference.
fdtd_status fdtd_solver_save_snapshot(fdtd_solver* s, const char* output_pattern, const char* numbering) {
    if (!s || !numbering) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    fdtd_status st = need_full_state(s);
    if (st != FDTD_OK) return st;
    const std::string pre = std::string("snapshot_") + numbering + "_";
    std::string path;
    if (!compose(output_pattern, pre + "x", path))
        return (set_error(s, "output pattern has no %s"), FDTD_ERR_INVALID_ARG);
    const long long N = s->ncell;
    const int ind = (int)((1 + s->step_index) % 3);
    std::vector<double> a;
    for (int d = 0; d < 3; ++d) {
        a.assign(N, 0.0);
        if ((st = fdtd_solver_get_field(s, FDTD_FIELD_PML_PX + d, a.data(), N)) != FDTD_OK) return st;
        compose(output_pattern, pre + "p_pml_" + std::to_string(d) + ".dat", path);
        if ((st = write_matrix(path, (int)N, 1, a.data())) != FDTD_OK) return st;
        const long long nv = s->vcount[d];
        a.assign(nv, 0.0);
        if ((st = fdtd_solver_get_field(s, FDTD_FIELD_VX + d, a.data(), nv)) != FDTD_OK) return st;
        compose(output_pattern, pre + "v_pml_" + std::to_string(d) + ".dat", path);
        if ((st = write_matrix(path, (int)nv, 1, a.data())) != FDTD_OK) return st;
        a.assign(N, 0.0);
        if (d == ind) st = fdtd_solver_get_field(s, FDTD_FIELD_PRESSURE, a.data(), N);
        else if (d == (ind + 2) % 3) st = fdtd_solver_get_field(s, FDTD_FIELD_PRESSURE_PREV, a.data(), N);
        if (st != FDTD_OK) return st;
        compose(output_pattern, pre + "p_collocated_" + std::to_string(d) + ".dat", path);
        if ((st = write_matrix(path, (int)N, 1, a.data())) != FDTD_OK) return st;
    }
    a.assign(N, 0.0);
    compose(output_pattern, pre + "p_pml_full.dat", path);
    if ((st = write_matrix(path, (int)N, 1, a.data())) != FDTD_OK) return st;
    compose(output_pattern, pre + "p_collocated_ind.dat", path);
    std::ofstream of(path.c_str());
    if (!of) return (set_error(s, "cannot open " + path), FDTD_ERR_IO);
    of << ind;
    of.close();
    return of ? FDTD_OK : (set_error(s, "short write to " + path), FDTD_ERR_IO);
}

// The inverse (no counterpart in the reference): the current and previous
// collocated pressures, split pressures and face velocities of a snapshot into
// this solve, whose grid must have the snapshot's sizes.  Time, step index and
// classification are the solver's own (load after fdtd_solver_reset to restart
// at the snapshot's time).
fdtd_status fdtd_solver_load_snapshot(fdtd_solver* s, const char* output_pattern, const char* numbering) {
    if (!s || !numbering) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    fdtd_status st = need_full_state(s);
    if (st != FDTD_OK) return st;
    const std::string pre = std::string("snapshot_") + numbering + "_";
    std::string path;
    if (!compose(output_pattern, pre + "p_collocated_ind.dat", path))
        return (set_error(s, "output pattern has no %s"), FDTD_ERR_INVALID_ARG);
    int ind = -1;
    {
        std::ifstream in(path.c_str());
        if (!(in >> ind) || ind < 0 || ind > 2) return (set_error(s, "cannot read " + path), FDTD_ERR_IO);
    }
    auto load = [&](const std::string& name, long long n, std::vector<double>& a) -> fdtd_status {
        compose(output_pattern, pre + name, path);
        int32_t r = 0, c = 0;
        a.assign(n, 0.0);
        fdtd_status e = fdtd_matrix_read(path.c_str(), &r, &c, nullptr, 0);
        if (e != FDTD_OK) return e;
        if ((long long)r * c != n) return (set_error(s, path + ": size does not match this grid"), FDTD_ERR_INVALID_ARG);
        return fdtd_matrix_read(path.c_str(), &r, &c, a.data(), n);
    };
    const long long N = s->ncell;
    std::vector<double> a;
    if ((st = load("p_collocated_" + std::to_string(ind) + ".dat", N, a)) != FDTD_OK) return st;
    if ((st = fdtd_solver_set_field(s, FDTD_FIELD_PRESSURE, a.data(), N)) != FDTD_OK) return st;
    if ((st = load("p_collocated_" + std::to_string((ind + 2) % 3) + ".dat", N, a)) != FDTD_OK) return st;
    if ((st = fdtd_solver_set_field(s, FDTD_FIELD_PRESSURE_PREV, a.data(), N)) != FDTD_OK) return st;
    for (int d = 0; d < 3; ++d) {
        if ((st = load("p_pml_" + std::to_string(d) + ".dat", N, a)) != FDTD_OK) return st;
        if ((st = fdtd_solver_set_field(s, FDTD_FIELD_PML_PX + d, a.data(), N)) != FDTD_OK) return st;
        if ((st = load("v_pml_" + std::to_string(d) + ".dat", s->vcount[d], a)) != FDTD_OK) return st;
        if ((st = fdtd_solver_set_field(s, FDTD_FIELD_VX + d, a.data(), s->vcount[d])) != FDTD_OK) return st;
    }
    return FDTD_OK;
}

// SaveSolverConfig's position files: pressure_vertex_position.dat (N x 3),
// velocity_<d>_vertex_position.dat, listening_position.dat (L x 3, none
// without listeners); cells in x-fastest order as the reference enumerates them.
fdtd_status fdtd_solver_save_config(fdtd_solver* s, const char* output_pattern) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    std::string path;
    if (!compose(output_pattern, "pressure_vertex_position.dat", path))
        return (set_error(s, "output pattern has no %s"), FDTD_ERR_INVALID_ARG);
    auto positions = [&](int face_dim, std::vector<double>& out, int& rows) {
        int ext[3] = {s->N[0], s->N[1], s->N[2]};
        if (face_dim >= 0) ext[face_dim] += 1;
        rows = ext[0] * ext[1] * ext[2];
        out.resize((size_t)rows * 3);
        size_t o = 0;
        for (int k = 0; k < ext[2]; ++k)
            for (int j = 0; j < ext[1]; ++j)
                for (int i = 0; i < ext[0]; ++i, o += 3) {
                    const int idx[3] = {i, j, k};
                    for (int d = 0; d < 3; ++d)
                        out[o + d] = (d == face_dim) ? s->tab[d].fpos[idx[d]] : s->tab[d].cpos[idx[d]];
                }
    };
    std::vector<double> a;
    int rows = 0;
    positions(-1, a, rows);
    fdtd_status st = write_matrix(path, rows, 3, a.data());
    if (st != FDTD_OK) return st;
    for (int d = 0; d < 3; ++d) {
        positions(d, a, rows);
        compose(output_pattern, "velocity_" + std::to_string(d) + "_vertex_position.dat", path);
        if ((st = write_matrix(path, rows, 3, a.data())) != FDTD_OK) return st;
    }
    if (s->L > 0) {
        compose(output_pattern, "listening_position.dat", path);
        if ((st = write_matrix(path, s->L, 3, s->listeners.data())) != FDTD_OK) return st;
    }
    return FDTD_OK;
}

// _SavePressureTimestep / _SaveVelocityTimestep: the current field as an
// (n x 1) matrix, cells (faces) in x-fastest order.
fdtd_status fdtd_solver_save_field_timestep(fdtd_solver* s, int32_t which, const char* path) {
    if (!s || !path || !(which == FDTD_FIELD_PRESSURE || (which >= FDTD_FIELD_VX && which <= FDTD_FIELD_VZ)))
        return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    int ext[3] = {s->N[0], s->N[1], s->N[2]};
    if (which >= FDTD_FIELD_VX) ext[which - FDTD_FIELD_VX] += 1;
    const long long n = (long long)ext[0] * ext[1] * ext[2];
    std::vector<double> dense(n), out(n);
    fdtd_status st = fdtd_solver_get_field(s, which, dense.data(), n);
    if (st != FDTD_OK) return st;
    long long o = 0;
    for (int k = 0; k < ext[2]; ++k)
        for (int j = 0; j < ext[1]; ++j)
            for (int i = 0; i < ext[0]; ++i, ++o) out[o] = dense[((long long)i * ext[1] + j) * ext[2] + k];
    return write_matrix(path, (int)n, 1, out.data());
}

}  // extern "C"
