// sifv_vtk_api.h -- internal interface between the VTK session
// (sifv_vtk.cpp, host only) and the device snapshot path in sifv_capi.cu.
#pragma once

#include <functional>
#include <string>

#include "sifv.h"

namespace sifv {

// Snapshot number for the next VTKSession::write (fileNum_++ of
// src/VTKSession.cpp:24-60); numbers are taken in call order.
int vtk_next_file(sifv_vtk_t* v);

// Queue work for the session's writer thread (FIFO, so .pvd entries keep the
// order of their numbers).  The job returns a SIFV_* status and an error
// message; the first failure is kept for sifv_vtk_flush.
void vtk_enqueue(sifv_vtk_t* v, std::function<int(std::string&)> job);

// Write snapshot `fileNum` at `time` from host fields (ghosted layout):
// the .vtr piece, the .pvtr meta-file and the .pvd entry.
int vtk_write_snapshot(sifv_vtk_t* v, int fileNum, double time, const sifv_vtk_fields_t* f, std::string& err);

// Session geometry: interior extents, ghost counts, dim, phases, IGR.
struct VtkLayout {
    int dim, nx, ny, nz, ngx, ngy, ngz, nPhases, useIGR;
};
const VtkLayout& vtk_layout(const sifv_vtk_t* v);

// Device staging owned by the capi side, released with the session.
void vtk_set_stage(sifv_vtk_t* v, void* stage, void (*release)(void*));
void* vtk_stage(sifv_vtk_t* v);

}  // namespace sifv
