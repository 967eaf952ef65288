// io.cu — host readers of the reference's mesh and current files, so that
// meshes and currents go from disk to the library's buffers without the
// reference's SurfMesh classes. Host code only (no device work); each reader
// counts when its output pointer is NULL, so a caller sizes the buffer with a
// first call and fills it with a second.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/bielcc_gpu.h"
#include "internal.h"

using namespace bielcc_gpu;

namespace {

int io_error(const std::string& msg) { return set_api_error(BIELCC_ERR_IO, msg.c_str()); }

}  // namespace

extern "C" {

// SurfMesh<CellQuad / CellTriangle>::ReadFromDatFile (mesh/surf_mesh.cpp:18-175):
// num_obj; per object kmod; per module "sign nfm . ." and nfm cells of n_vert
// vertices (x y z each); then the separation lines (count, segments), which
// are not cells and are skipped.
int bielcc_read_mesh_dat(const char* path, int n_vert, int* n_cells, double* cells) {
    if (!path || !n_cells || (n_vert != 3 && n_vert != 4))
        return set_api_error(BIELCC_ERR_ARG, "read_mesh_dat: path, n_cells and n_vert 3 or 4 required");
    std::ifstream fin(path);
    if (!fin.is_open()) return io_error(std::string("cannot open ") + path);
    int n_obj = 0;
    if (!(fin >> n_obj) || n_obj < 0) return io_error("read_mesh_dat: bad object count");
    long long total = 0;
    const int cap = cells ? *n_cells : 0;
    for (int o = 0; o < n_obj; o++) {
        int kmod = 0;
        if (!(fin >> kmod) || kmod < 0) return io_error("read_mesh_dat: bad module count");
        for (int j = 0; j < kmod; j++) {
            int sign, nfm, u1, u2;
            if (!(fin >> sign >> nfm >> u1 >> u2) || nfm < 0) return io_error("read_mesh_dat: bad module header");
            for (int c = 0; c < nfm; c++, total++) {
                double v[12];
                for (int i = 0; i < 3 * n_vert; i++)
                    if (!(fin >> v[i])) return io_error("read_mesh_dat: unexpected end of cell data");
                if (cells) {
                    if (total >= cap) return set_api_error(BIELCC_ERR_ARG, "read_mesh_dat: buffer too small");
                    memcpy(cells + total * 3 * n_vert, v, sizeof(double) * 3 * n_vert);
                }
            }
        }
    }
    *n_cells = (int)total;
    return BIELCC_OK;
}

// SurfMesh<...>::ReadFromVtkFile + FillMeshFromVTK (mesh/surf_mesh.h:382-560,
// mesh/surf_mesh.cpp:195-290): legacy ASCII VTK, POINTS and POLYGONS (POLYDATA)
// or CELLS (UNSTRUCTURED_GRID); polygons with exactly n_vert vertices become
// cells in file order, others are skipped (their count in *n_skipped, may be
// NULL); an index outside the point list, and a file without any polygon of
// n_vert vertices, are errors, as the reference throws for both.
int bielcc_read_mesh_vtk(const char* path, int n_vert, int* n_cells, double* cells, int* n_skipped) {
    if (!path || !n_cells || (n_vert != 3 && n_vert != 4))
        return set_api_error(BIELCC_ERR_ARG, "read_mesh_vtk: path, n_cells and n_vert 3 or 4 required");
    std::ifstream fin(path);
    if (!fin.is_open()) return io_error(std::string("cannot open ") + path);
    std::vector<double> pts;
    std::vector<std::vector<int>> polys;
    std::string line;
    while (std::getline(fin, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream iss(line);
        std::string kw;
        iss >> kw;
        if (kw == "POINTS") {
            long long np = 0;
            iss >> np;
            if (np < 0) return io_error("read_mesh_vtk: bad POINTS count");
            pts.resize(3 * np);
            for (long long i = 0; i < 3 * np; i++)
                if (!(fin >> pts[i])) return io_error("read_mesh_vtk: unexpected end of points");
        } else if (kw == "POLYGONS" || kw == "CELLS") {
            long long nc = 0, tot = 0;
            iss >> nc >> tot;
            if (nc < 0) return io_error("read_mesh_vtk: bad " + kw + " count");
            polys.resize(nc);
            for (long long i = 0; i < nc; i++) {
                int n = 0;
                if (!(fin >> n) || n < 0) return io_error("read_mesh_vtk: bad polygon size");
                polys[i].resize(n);
                for (int j = 0; j < n; j++)
                    if (!(fin >> polys[i][j])) return io_error("read_mesh_vtk: unexpected end of polygons");
            }
        } else if (kw == "CELL_DATA" || kw == "POINT_DATA") {
            break;  // attributes follow: the geometry is complete
        }
    }
    if (pts.empty() || polys.empty()) return io_error("read_mesh_vtk: no points or cells");
    const long long np = (long long)pts.size() / 3;
    const int cap = cells ? *n_cells : 0;
    int count = 0, skipped = 0;
    for (const auto& p : polys) {
        if ((int)p.size() != n_vert) {
            skipped++;
            continue;
        }
        for (int v = 0; v < n_vert; v++)
            if (p[v] < 0 || p[v] >= np) return io_error("read_mesh_vtk: point index out of range");
        if (cells) {
            if (count >= cap) return set_api_error(BIELCC_ERR_ARG, "read_mesh_vtk: buffer too small");
            for (int v = 0; v < n_vert; v++)
                for (int g = 0; g < 3; g++) cells[((size_t)count * n_vert + v) * 3 + g] = pts[3 * (size_t)p[v] + g];
        }
        count++;
    }
    if (n_skipped) *n_skipped = skipped;
    // FillMeshFromVTK throws when no polygon has the cell's vertex count
    if (count == 0) return io_error("read_mesh_vtk: no polygon with " + std::to_string(n_vert) + " vertices");
    *n_cells = count;
    return BIELCC_OK;
}

// SurfaceCurrentsC_fromFiles (electrodynamics/currents.cpp:74-109): two files,
// real and imaginary parts, each "n1 n2" then n1*n2 rows of three numbers;
// J[i] = (re + i im) per component, interleaved complex [n][3].
int bielcc_read_currents(const char* path_re, const char* path_im, int* n, double* J) {
    if (!path_re || !path_im || !n) return set_api_error(BIELCC_ERR_ARG, "read_currents: paths and n required");
    std::ifstream fr(path_re), fi(path_im);
    if (!fr.is_open() || !fi.is_open()) return io_error("read_currents: cannot open the current files");
    long long a1, a2, b1, b2;
    if (!(fr >> a1 >> a2) || !(fi >> b1 >> b2)) return io_error("read_currents: bad header");
    if (a1 != b1 || a2 != b2 || a1 < 0 || a2 < 0)
        return io_error("read_currents: the real and imaginary files disagree in size");
    const long long cnt = a1 * a2;
    if (J) {
        if (cnt > *n) return set_api_error(BIELCC_ERR_ARG, "read_currents: buffer too small");
        for (long long i = 0; i < cnt; i++)
            for (int g = 0; g < 3; g++) {
                double re, im;
                if (!(fr >> re) || !(fi >> im)) return io_error("read_currents: unexpected end of data");
                J[(i * 3 + g) * 2] = re;
                J[(i * 3 + g) * 2 + 1] = im;
            }
    }
    *n = (int)cnt;
    return BIELCC_OK;
}

}  // extern "C"
