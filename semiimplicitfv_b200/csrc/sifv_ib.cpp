// sifv_ib.cpp -- immersed-boundary set-up (ImmersedBoundaryMethod::
// classifyCells, src/ImmersedBoundary.cpp:190-392) on the host, once per
// body set: the classification is a one-off geometric query over the mesh;
// the per-stage ghost-cell fill that it feeds runs on the device.
//
// Cells whose centroid lies inside a body (signed distance < 0) are dead;
// a dead cell with a fluid face neighbour becomes a ghost cell.  Each ghost
// cell mirrors its centroid through the closest surface point and takes a
// bi/trilinear stencil of the cells around that image point, falling back to
// one fluid cell of the stencil when the stencil touches the body.  The
// arithmetic follows the reference expression by expression (no
// contraction: this file is compiled with -ffp-contract=off).
#include <algorithm>
#include <cmath>

#include "sifv_ib_api.h"

namespace sifv {
namespace {

double smaxd(double a, double b) { return (a < b) ? b : a; }
double smind(double a, double b) { return (b < a) ? b : a; }
double clampd(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
double sgn(double v) { return (v >= 0) ? 1.0 : -1.0; }

// cross-section coordinates of a cylinder along `axis`
void plane(int axis, double x, double y, double z, double& p0, double& p1) {
    if (axis == 0) { p0 = y; p1 = z; }
    else if (axis == 1) { p0 = x; p1 = z; }
    else { p0 = x; p1 = y; }
}

// IBCircle / IBRectangle / IBCylinder / IBRectangularPrism (src/ImmersedBoundary.cpp:9-180)
double sdf(void* user, int bi, double x, double y, double z) {
    const sifv_ib_body_t& b = static_cast<const sifv_ib_body_t*>(user)[bi];
    const double* p = b.p;
    if (b.shape == SIFV_IB_CIRCLE) {
        double dx = x - p[0], dy = y - p[1];
        return std::sqrt(dx * dx + dy * dy) - p[2];
    }
    if (b.shape == SIFV_IB_RECTANGLE) {
        double qx = std::fabs(x - p[0]) - p[2], qy = std::fabs(y - p[1]) - p[3];
        double out = std::sqrt(smaxd(qx, 0.0) * smaxd(qx, 0.0) + smaxd(qy, 0.0) * smaxd(qy, 0.0));
        return out + smind(smaxd(qx, qy), 0.0);
    }
    if (b.shape == SIFV_IB_CYLINDER) {
        double p0, p1;
        plane(b.axis, x, y, z, p0, p1);
        double d0 = p0 - p[0], d1 = p1 - p[1];
        return std::sqrt(d0 * d0 + d1 * d1) - p[2];
    }
    double qx = std::fabs(x - p[0]) - p[3], qy = std::fabs(y - p[1]) - p[4], qz = std::fabs(z - p[2]) - p[5];
    double out = std::sqrt(smaxd(qx, 0.0) * smaxd(qx, 0.0) + smaxd(qy, 0.0) * smaxd(qy, 0.0) +
                           smaxd(qz, 0.0) * smaxd(qz, 0.0));
    return out + smind(smaxd(smaxd(qx, qy), qz), 0.0);
}

void closest(void* user, int bi, double x, double y, double z, double o[3]) {
    const sifv_ib_body_t& b = static_cast<const sifv_ib_body_t*>(user)[bi];
    const double* p = b.p;
    if (b.shape == SIFV_IB_CIRCLE) {
        double dx = x - p[0], dy = y - p[1];
        double dist = std::sqrt(dx * dx + dy * dy);
        if (dist < 1e-14) {
            o[0] = p[0] + p[2]; o[1] = p[1]; o[2] = 0.0;
            return;
        }
        double s = p[2] / dist;
        o[0] = p[0] + dx * s; o[1] = p[1] + dy * s; o[2] = 0.0;
    } else if (b.shape == SIFV_IB_RECTANGLE) {
        double dx = x - p[0], dy = y - p[1];
        double qx = clampd(dx, -p[2], p[2]), qy = clampd(dy, -p[3], p[3]);
        if (std::fabs(dx) <= p[2] && std::fabs(dy) <= p[3]) {   // inside: push to the nearer side
            if (p[2] - std::fabs(dx) < p[3] - std::fabs(dy)) qx = (dx >= 0) ? p[2] : -p[2];
            else qy = (dy >= 0) ? p[3] : -p[3];
        }
        o[0] = p[0] + qx; o[1] = p[1] + qy; o[2] = 0.0;
    } else if (b.shape == SIFV_IB_CYLINDER) {
        double p0, p1;
        plane(b.axis, x, y, z, p0, p1);
        double d0 = p0 - p[0], d1 = p1 - p[1];
        double dist = std::sqrt(d0 * d0 + d1 * d1);
        double q0, q1;
        if (dist < 1e-14) {
            q0 = p[0] + p[2];
            q1 = p[1];
        } else {
            double s = p[2] / dist;
            q0 = p[0] + d0 * s;
            q1 = p[1] + d1 * s;
        }
        if (b.axis == 0) { o[0] = x; o[1] = q0; o[2] = q1; }
        else if (b.axis == 1) { o[0] = q0; o[1] = y; o[2] = q1; }
        else { o[0] = q0; o[1] = q1; o[2] = z; }
    } else {
        double dx = x - p[0], dy = y - p[1], dz = z - p[2];
        double qx = clampd(dx, -p[3], p[3]), qy = clampd(dy, -p[4], p[4]), qz = clampd(dz, -p[5], p[5]);
        if (std::fabs(dx) <= p[3] && std::fabs(dy) <= p[4] && std::fabs(dz) <= p[5]) {
            double ex = p[3] - std::fabs(dx), ey = p[4] - std::fabs(dy), ez = p[5] - std::fabs(dz);
            if (ex <= ey && ex <= ez) qx = (dx >= 0) ? p[3] : -p[3];
            else if (ey <= ex && ey <= ez) qy = (dy >= 0) ? p[4] : -p[4];
            else qz = (dz >= 0) ? p[5] : -p[5];
        }
        o[0] = p[0] + qx; o[1] = p[1] + qy; o[2] = p[2] + qz;
    }
}

void normal(void* user, int bi, double x, double y, double z, double o[3]) {
    const sifv_ib_body_t& b = static_cast<const sifv_ib_body_t*>(user)[bi];
    const double* p = b.p;
    if (b.shape == SIFV_IB_CIRCLE) {
        double dx = x - p[0], dy = y - p[1];
        double dist = std::sqrt(dx * dx + dy * dy);
        if (dist < 1e-14) {
            o[0] = 1.0; o[1] = 0.0; o[2] = 0.0;
            return;
        }
        o[0] = dx / dist; o[1] = dy / dist; o[2] = 0.0;
    } else if (b.shape == SIFV_IB_RECTANGLE) {
        double cp[3];
        closest(user, bi, x, y, z, cp);
        double dx = cp[0] - p[0], dy = cp[1] - p[1];
        bool onX = std::fabs(std::fabs(dx) - p[2]) < 1e-12, onY = std::fabs(std::fabs(dy) - p[3]) < 1e-12;
        if (onX && !onY) { o[0] = sgn(dx); o[1] = 0.0; o[2] = 0.0; }
        else if (onY && !onX) { o[0] = 0.0; o[1] = sgn(dy); o[2] = 0.0; }
        else {   // a corner: the diagonal
            double len = std::sqrt(2.0);
            o[0] = sgn(dx) / len; o[1] = sgn(dy) / len; o[2] = 0.0;
        }
    } else if (b.shape == SIFV_IB_CYLINDER) {
        double p0, p1;
        plane(b.axis, x, y, z, p0, p1);
        double d0 = p0 - p[0], d1 = p1 - p[1];
        double dist = std::sqrt(d0 * d0 + d1 * d1);
        double n0 = 1.0, n1 = 0.0;
        if (!(dist < 1e-14)) {
            n0 = d0 / dist;
            n1 = d1 / dist;
        }
        if (b.axis == 0) { o[0] = 0.0; o[1] = n0; o[2] = n1; }
        else if (b.axis == 1) { o[0] = n0; o[1] = 0.0; o[2] = n1; }
        else { o[0] = n0; o[1] = n1; o[2] = 0.0; }
    } else {
        double cp[3];
        closest(user, bi, x, y, z, cp);
        double d[3] = {cp[0] - p[0], cp[1] - p[1], cp[2] - p[2]};
        double nv[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 3; ++a)
            if (std::fabs(std::fabs(d[a]) - p[3 + a]) < 1e-12) nv[a] = sgn(d[a]);
        double len = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
        if (len < 1e-14) {
            o[0] = 1.0; o[1] = 0.0; o[2] = 0.0;
            return;
        }
        o[0] = nv[0] / len; o[1] = nv[1] / len; o[2] = nv[2] / len;
    }
}

// lower cell of the centroid interval holding `v` (findCell, 190-214)
int find_cell(const std::vector<double>& c, double v) {
    const int n = (int)c.size();
    if (n <= 1) return 0;
    if (v <= c[0]) return 0;
    if (v >= c[n - 1]) return std::max(0, n - 2);
    for (int i = 0; i < n - 1; ++i)
        if (v >= c[i] && v < c[i + 1]) return i;
    return std::max(0, n - 2);
}

double frac(double v, double c0, double c1) {
    double d = c1 - c0;
    return (d > 1e-14) ? clampd((v - c0) / d, 0.0, 1.0) : 0.0;
}

}  // namespace

void ib_builtin_shapes(const sifv_ib_body_t* bodies, sifv_ib_shapes_t& out) {
    out.user = const_cast<sifv_ib_body_t*>(bodies);
    out.signedDistance = sdf;
    out.closestPoint = closest;
    out.outwardNormal = normal;
}

void ib_classify(const IbGeometry& g, int nBodies, const int* wall, const sifv_ib_shapes_t& s, IbTable& t) {
    auto idx = [&](int i, int j, int k) {
        return (long long)(i + g.ngx) + g.nxT * ((long long)(j + g.ngy) + g.nyT * (long long)(k + g.ngz));
    };
    t = IbTable();
    t.type.assign(g.ncells, SIFV_CELL_FLUID);
    std::vector<int> owner(g.ncells, -1);
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
                for (int b = 0; b < nBodies; ++b)
                    if (s.signedDistance(s.user, b, g.cx[i], g.cy[j], g.cz[k]) < 0) {
                        t.type[idx(i, j, k)] = SIFV_CELL_DEAD;
                        owner[idx(i, j, k)] = b;
                        break;
                    }
    auto fluid = [&](int i, int j, int k) { return t.type[idx(i, j, k)] == SIFV_CELL_FLUID; };
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                if (t.type[idx(i, j, k)] != SIFV_CELL_DEAD) continue;
                bool f = (i > 0 && fluid(i - 1, j, k)) || (i < g.nx - 1 && fluid(i + 1, j, k));
                if (g.dim >= 2) f = f || (j > 0 && fluid(i, j - 1, k)) || (j < g.ny - 1 && fluid(i, j + 1, k));
                if (g.dim >= 3) f = f || (k > 0 && fluid(i, j, k - 1)) || (k < g.nz - 1 && fluid(i, j, k + 1));
                if (f) t.type[idx(i, j, k)] = SIFV_CELL_GHOST;
            }
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                const long long c = idx(i, j, k);
                if (t.type[c] != SIFV_CELL_GHOST) continue;
                const int b = owner[c];
                const double xG = g.cx[i], yG = g.cy[j], zG = g.cz[k];
                double cp[3], nv[3];
                s.closestPoint(s.user, b, xG, yG, zG, cp);
                s.outwardNormal(s.user, b, xG, yG, zG, nv);
                const double xI = 2.0 * cp[0] - xG, yI = 2.0 * cp[1] - yG, zI = 2.0 * cp[2] - zG;
                // buildInterpStencil (216-300)
                const int i0 = find_cell(g.cx, xI);
                const int j0 = (g.dim >= 2) ? find_cell(g.cy, yI) : 0;
                const int k0 = (g.dim >= 3) ? find_cell(g.cz, zI) : 0;
                const int i1 = std::min(i0 + 1, g.nx - 1), j1 = std::min(j0 + 1, g.ny - 1),
                          k1 = std::min(k0 + 1, g.nz - 1);
                const double tx = frac(xI, g.cx[i0], g.cx[i1]);
                long long cs[8];
                double ws[8];
                int n;
                if (g.dim == 1) {
                    n = 2;
                    cs[0] = idx(i0, 0, 0); cs[1] = idx(i1, 0, 0);
                    ws[0] = 1.0 - tx; ws[1] = tx;
                } else {
                    const double ty = frac(yI, g.cy[j0], g.cy[j1]);
                    if (g.dim == 2) {
                        n = 4;
                        cs[0] = idx(i0, j0, 0); cs[1] = idx(i1, j0, 0); cs[2] = idx(i0, j1, 0); cs[3] = idx(i1, j1, 0);
                        ws[0] = (1.0 - tx) * (1.0 - ty); ws[1] = tx * (1.0 - ty);
                        ws[2] = (1.0 - tx) * ty; ws[3] = tx * ty;
                    } else {
                        const double tz = frac(zI, g.cz[k0], g.cz[k1]);
                        n = 8;
                        const int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
                        for (int q = 0; q < 8; ++q) cs[q] = idx(ii[q & 1], jj[(q >> 1) & 1], kk[q >> 2]);
                        ws[0] = (1.0 - tx) * (1.0 - ty) * (1.0 - tz); ws[1] = tx * (1.0 - ty) * (1.0 - tz);
                        ws[2] = (1.0 - tx) * ty * (1.0 - tz); ws[3] = tx * ty * (1.0 - tz);
                        ws[4] = (1.0 - tx) * (1.0 - ty) * tz; ws[5] = tx * (1.0 - ty) * tz;
                        ws[6] = (1.0 - tx) * ty * tz; ws[7] = tx * ty * tz;
                    }
                }
                bool allFluid = true;
                for (int q = 0; q < n; ++q) allFluid = allFluid && t.type[cs[q]] == SIFV_CELL_FLUID;
                if (!allFluid) {   // one fluid cell of the stencil (the first), else its first cell
                    long long f = cs[0];
                    for (int q = 0; q < n; ++q)
                        if (t.type[cs[q]] == SIFV_CELL_FLUID) {
                            f = cs[q];
                            break;
                        }
                    n = 1;
                    cs[0] = f;
                    ws[0] = 1.0;
                }
                for (int q = 0; q < n; ++q)
                    if (t.type[cs[q]] == SIFV_CELL_GHOST) t.sequential = 1;
                t.cell.push_back(c);
                t.wall.push_back(wall[b]);
                t.n.push_back(n);
                for (int a = 0; a < 3; ++a) t.normal.push_back(nv[a]);
                for (int q = 0; q < 8; ++q) {
                    t.interp.push_back(q < n ? cs[q] : cs[0]);
                    t.w.push_back(q < n ? ws[q] : 0.0);
                }
            }
}

}  // namespace sifv
