// mesh.cu — per-mesh preparation on the device: the per-cell geometry rows and
// the x-independent quadrature node tables. The reference recomputes this
// geometry inside every (point, cell) call (integral_universal.h:58-93,
// element_geom.cpp); here it is computed once per mesh and split.
#include "internal.h"
#include "ops.cuh"

namespace bielcc_gpu {

// One thread per cell: centre (get_center_mass), diam (get_diam), normal
// (norm_func), tangent basis and area as CellFill stores them
// (mesh/cell.cpp:8-51 quad, :60-99 triangle), and the vertex radius rho.
__global__ void cell_geometry_kernel(const double* __restrict__ verts, int nv, int n_cells, CellGeo* __restrict__ geo) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    DCell cl;
    cl.nv = nv;
    for (int v = 0; v < nv; v++)
        for (int g = 0; g < 3; g++) cl.v[v][g] = verts[((size_t)c * nv + v) * 3 + g];
    CellGeo o;
    cell_centre(cl, o.c);
    o.diam = cell_diam(cl);
    cell_normal(cl, o.n);
    double nrm[3], base[3], len;
    if (nv == 4) {
        double ma[3], mb[3], mc[3], md[3], bd[3];
        for (int i = 0; i < 3; i++) {
            ma[i] = (cl.v[0][i] + cl.v[1][i]) / 2.0;
            mb[i] = (cl.v[1][i] + cl.v[2][i]) / 2.0;
            mc[i] = (cl.v[2][i] + cl.v[3][i]) / 2.0;
            md[i] = (cl.v[3][i] + cl.v[0][i]) / 2.0;
            base[i] = mc[i] - ma[i];
            bd[i] = md[i] - mb[i];
        }
        cross3(base, bd, nrm);
        len = len3(nrm);
        o.area = len;
    } else {
        double ac[3];
        for (int i = 0; i < 3; i++) { base[i] = cl.v[1][i] - cl.v[0][i]; ac[i] = cl.v[2][i] - cl.v[0][i]; }
        cross3(base, ac, nrm);
        len = len3(nrm);
        o.area = len / 2;
    }
    for (int i = 0; i < 3; i++) nrm[i] /= len;
    len = len3(base);
    for (int i = 0; i < 3; i++) o.t1[i] = base[i] / len;
    cross3(nrm, o.t1, o.t2);
    len = len3(o.t2);
    for (int i = 0; i < 3; i++) o.t2[i] /= len;
    double rho = 0.;
    for (int v = 0; v < nv; v++) rho = fmax(rho, dist3(cl.v[v], o.c));
    o.rho = rho;
    o.pad = 0.;
    geo[c] = o;
}

// One thread per cell: the n^2 nodes of the midpoint rule in the reference's
// visiting order (quad: i-major over the bilinear split, integral_universal.h:59-93;
// triangle: lower then upper sub-triangle per (i, j), :166-193). FP64 rows
// hold (y, weight); FP32 rows hold (y - centre, weight). Triangle weights are
// area / n / n (the reference scales the sum once; same value up to rounding).
// out32 and rho32 may be null (an FP64-only table).
__global__ void node_table_kernel(const double* __restrict__ verts, const CellGeo* __restrict__ geo, int nv,
                                  int n_cells, int n, double4* __restrict__ out64, float4* __restrict__ out32,
                                  float* __restrict__ rho32) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    double v[4][3];
    for (int a = 0; a < nv; a++)
        for (int g = 0; g < 3; g++) v[a][g] = verts[((size_t)c * nv + a) * 3 + g];
    const double* ctr = geo[c].c;
    size_t base = (size_t)c * n * n;
    int idx = 0;
    float rmax = 0.f;
    auto emit = [&](const double* y, double w) {
        out64[base + idx] = make_double4(y[0], y[1], y[2], w);
        float dx = (float)(y[0] - ctr[0]), dy = (float)(y[1] - ctr[1]), dz = (float)(y[2] - ctr[2]);
        if (out32) out32[base + idx] = make_float4(dx, dy, dz, (float)w);
        rmax = fmaxf(rmax, sqrtf(dx * dx + dy * dy + dz * dz));
        idx++;
    };
    if (nv == 4) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double y[3], s;
                quad_node(v, i, j, n, y, &s);
                emit(y, s);
            }
    } else {
        double area = tri_area(v[0], v[1], v[2]);
        double w = area / (double)n / (double)n;
        double pv[3], qv[3], rv[3];
        for (int k = 0; k < 3; k++) {
            pv[k] = (v[1][k] - v[0][k]) / n;
            qv[k] = (v[2][k] - v[0][k]) / n;
            rv[k] = (v[2][k] - v[1][k]) / n;
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n - i; j++) {
                double B[3], y[3];
                for (int k = 0; k < 3; k++) {
                    B[k] = v[0][k] + (i + 1) * pv[k] + j * qv[k];
                    double A = B[k] - pv[k];
                    y[k] = (B[k] + A + (A + qv[k])) / 3.0;
                }
                emit(y, w);
                if (j < n - 1 - i) {
                    for (int k = 0; k < 3; k++) y[k] = (B[k] + (B[k] + rv[k]) + (B[k] + qv[k])) / 3.0;
                    emit(y, w);
                }
            }
    }
    if (rho32) rho32[c] = rmax;
}

cudaError_t launch_cell_geometry(const double* verts, int nv, int n_cells, CellGeo* geo, cudaStream_t s) {
    if (n_cells <= 0) return cudaSuccess;
    cell_geometry_kernel<<<(n_cells + 127) / 128, 128, 0, s>>>(verts, nv, n_cells, geo);
    return cudaGetLastError();
}

cudaError_t launch_node_tables(const double* verts, const CellGeo* geo, int nv, int n_cells, int n, double4* nodes64,
                               float4* nodes32, float* rho32, cudaStream_t s) {
    if (n_cells <= 0) return cudaSuccess;
    node_table_kernel<<<(n_cells + 63) / 64, 64, 0, s>>>(verts, geo, nv, n_cells, n, nodes64, nodes32, rho32);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
