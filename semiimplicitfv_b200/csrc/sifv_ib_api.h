// sifv_ib_api.h -- immersed-boundary set-up on the host (sifv_ib.cpp): the
// cell classification and ghost-cell stencils that the device kernels use.
#pragma once

#include <vector>

#include "sifv.h"

namespace sifv {

// Interior cell centroids per axis and the context's index layout.
struct IbGeometry {
    int dim, nx, ny, nz, ngx, ngy, ngz;
    long long nxT, nyT;
    size_t ncells;
    std::vector<double> cx, cy, cz;
};

// CellType per cell and the ghost-cell list in (k, j, i) order.
struct IbTable {
    std::vector<unsigned char> type;
    std::vector<long long> cell, interp;   // interp: 8 per entry
    std::vector<int> wall, n;
    std::vector<double> normal, w;         // normal: 3 per entry, w: 8 per entry
    int sequential = 0;
};

// The four body classes of the reference as shape queries (user = the body array).
void ib_builtin_shapes(const sifv_ib_body_t* bodies, sifv_ib_shapes_t& out);
// ImmersedBoundaryMethod::classifyCells over any shape queries.
void ib_classify(const IbGeometry& g, int nBodies, const int* wall, const sifv_ib_shapes_t& s, IbTable& t);

}  // namespace sifv
