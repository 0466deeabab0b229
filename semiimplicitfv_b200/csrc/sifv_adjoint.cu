// sifv_adjoint.cu -- launchers of the discrete adjoint and tangent kernels.
#include "sifv_adjoint.cuh"

namespace sifv {

namespace {

unsigned nblocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

long long nfaces(const Params& P, int d) {
    return (long long)(P.nx + (d == 0)) * (P.ny + (d == 1)) * (P.nz + (d == 2));
}

template <int DIM, typename S>
void adj_faces(const AdjArgs& A, cudaStream_t s) {
    k_adj_face<0, DIM, S><<<nblocks(nfaces(A.P, 0), 128), 128, 0, s>>>(A);
    if (DIM >= 2) k_adj_face<(DIM >= 2 ? 1 : 0), DIM, S><<<nblocks(nfaces(A.P, 1), 128), 128, 0, s>>>(A);
    if (DIM >= 3) k_adj_face<(DIM >= 3 ? 2 : 0), DIM, S><<<nblocks(nfaces(A.P, 2), 128), 128, 0, s>>>(A);
}

template <int DIM>
void adj_stage(const AdjArgs& A, cudaStream_t s) {
    if (A.fp32) adj_faces<DIM, float>(A, s);
    else adj_faces<DIM, double>(A, s);
    const long long n = (long long)A.P.nx * A.P.ny * A.P.nz;
    k_adj_cell<DIM><<<nblocks(n, 128), 128, 0, s>>>(A);
}

template <int DIM>
void tan_faces(const AdjArgs& A, cudaStream_t s) {
    const long long ne = (long long)A.P.nxT * A.P.nyT * A.P.nzT;
    k_tan_prim<DIM><<<nblocks(ne, 256), 256, 0, s>>>(A);
    k_tan_face<0, DIM><<<nblocks(nfaces(A.P, 0), 128), 128, 0, s>>>(A);
    if (DIM >= 2) k_tan_face<(DIM >= 2 ? 1 : 0), DIM><<<nblocks(nfaces(A.P, 1), 128), 128, 0, s>>>(A);
    if (DIM >= 3) k_tan_face<(DIM >= 3 ? 2 : 0), DIM><<<nblocks(nfaces(A.P, 2), 128), 128, 0, s>>>(A);
}

__global__ void k_zero_ghosts(Params P, double* f) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ext_coords(P, t, i, j, k)) return;
    if (!is_interior(P, i, j, k)) f[cidx(P, i, j, k)] = 0.0;
}

}  // namespace

int adjoint_stage(const AdjArgs& A, cudaStream_t s) {
    switch (A.P.dim) {
        case 1: adj_stage<1>(A, s); break;
        case 2: adj_stage<2>(A, s); break;
        default: adj_stage<3>(A, s); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int tangent_faces(const AdjArgs& A, cudaStream_t s) {
    switch (A.P.dim) {
        case 1: tan_faces<1>(A, s); break;
        case 2: tan_faces<2>(A, s); break;
        default: tan_faces<3>(A, s); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int tangent_update(const AdjArgs& A, int save, cudaStream_t s) {
    const long long n = (long long)A.P.nx * A.P.ny * A.P.nz;
    switch (A.P.dim) {
        case 1: k_tan_update<1><<<nblocks(n, 256), 256, 0, s>>>(A, save); break;
        case 2: k_tan_update<2><<<nblocks(n, 256), 256, 0, s>>>(A, save); break;
        default: k_tan_update<3><<<nblocks(n, 256), 256, 0, s>>>(A, save); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int zero_ghosts(const Params& P, double* f, cudaStream_t s) {
    const long long ne = (long long)P.nxT * P.nyT * P.nzT;
    k_zero_ghosts<<<nblocks(ne, 256), 256, 0, s>>>(P, f);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace sifv
