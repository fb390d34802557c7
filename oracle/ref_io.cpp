// Reference harness, geometry files -- TEST INFRASTRUCTURE (linked into
// oracle/_ref/libmarqov_ref.so; used by tests/ only).
//
// Runs the reference's own save_geometry / import_geometry_ncoords /
// import_geometry (src/lattice/util/io.h:34-126) and GraphFromCSV's use of
// them (src/lattice/graph_from_csv.h:40-44) on plain arrays.
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "lattice/util/io.h"

namespace {
// a lattice over CSR arrays with the reference's lattice interface
struct ArrayGrid {
    int n;
    const int* rp;
    const int* ci;
    int nc;
    const double* crd;
    int size() const { return n; }
    std::vector<int> nbrs(int, int i) const { return std::vector<int>(ci + rp[i], ci + rp[i + 1]); }
    std::vector<double> crds(int i) const { return std::vector<double>(crd + (size_t)i * nc, crd + (size_t)(i + 1) * nc); }
};
}  // namespace

extern "C" int ref_save_geometry(int n, const int* rp, const int* ci, int nc, const double* crd, const char* path)
{
    ArrayGrid g{n, rp, ci, nc, crd};
    save_geometry(g, std::string(path));
    return 0;
}

// GraphFromCSV(path) with import_geometry's idxoffs.  Call with null arrays
// for the sizes (sites, neighbour entries, coordinate values, ncoords), then
// with arrays of those sizes: rp [n + 1], ci [nnz], ncrd [n] coordinates per
// site, crd [coordinate values].  Returns -1 where the reference throws.
extern "C" int ref_import_geometry(const char* path, int idxoffs, int* n, int* nnz, int* ncrd_total, int* ncoords,
                                   int* rp, int* ci, int* ncrd, double* crd)
{
    try {
        std::vector<std::vector<double>> grid;
        std::vector<std::vector<int>> nb;
        const int c = import_geometry_ncoords(std::string(path));
        const int np = import_geometry(std::string(path), grid, nb, c, idxoffs);
        int e = 0, v = 0;
        for (int i = 0; i < np; ++i) {
            e += (int)nb[i].size();
            v += (int)grid[i].size();
        }
        *n = np;
        *nnz = e;
        *ncrd_total = v;
        *ncoords = c;
        if (!rp) return 0;
        rp[0] = 0;
        int pe = 0, pv = 0;
        for (int i = 0; i < np; ++i) {
            for (int j : nb[i]) ci[pe++] = j;
            rp[i + 1] = pe;
            ncrd[i] = (int)grid[i].size();
            for (double x : grid[i]) crd[pv++] = x;
        }
        return 0;
    } catch (...) {
        return -1;
    }
}
