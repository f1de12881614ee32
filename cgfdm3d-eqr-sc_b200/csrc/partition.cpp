// Domain decomposition of a model: one part of a PX x PY x PZ grid of
// sub-domains, as the reference's MPI ranks hold them (src/init_grid.cpp,
// src/init_MPI.cpp), built by slicing the global model.  A part's padded
// arrays are the global arrays over the part's interior plus 3 cells on
// each side, so every value a part reads inside its own interior equals the
// global one; the halos at internal faces are refreshed by halo exchange
// while stepping (csrc/halo.cu).
#include <algorithm>
#include <string>
#include <vector>

#include "model.hpp"

namespace cgfdm {

void part_extent(int N, int n, int c, int *lo, int *len)
{
    const int base = N / n, rem = N % n;
    *len = base + (c < rem ? 1 : 0);
    *lo = c * base + std::min(c, rem);
}

int slice_model(const Model &G, const int parts[3], const int coord[3], Model &m, std::string &err)
{
    if (G.p.scheme != SCHEME_CGFDM) {
        err = "domain decomposition is built for the CGFDM scheme";
        return ST_OPTIONS;
    }
    const int Nn[3] = {G.g.nx, G.g.ny, G.g.nz};
    int lo[3], n[3];
    for (int a = 0; a < 3; a++) {
        if (parts[a] < 1 || coord[a] < 0 || coord[a] >= parts[a]) {
            err = "bad decomposition or part coordinate";
            return ST_ARG;
        }
        part_extent(Nn[a], parts[a], coord[a], &lo[a], &n[a]);
        // the 3-cell halo must come from one neighbour, and a PML slab must
        // lie inside one part (src/pml_deriv.cpp:55-85 checks nPML < n)
        if (n[a] < 2 * HALO) {
            err = "a part is thinner than 6 cells";
            return ST_OPTIONS;
        }
    }
    m.p = G.p;
    m.NT = G.NT;
    m.g = G.g;
    Grid &g = m.g;
    g.nx = n[0], g.ny = n[1], g.nz = n[2];
    g._nx_ = n[0] + 2 * HALO, g._ny_ = n[1] + 2 * HALO, g._nz_ = n[2] + 2 * HALO;
    g._nx = n[0] + HALO, g._ny = n[1] + HALO, g._nz = n[2] + HALO;
    for (int a = 0; a < 3; a++) {
        m.part_lo[a] = lo[a];
        m.parts[a] = parts[a];
        m.part_coord[a] = coord[a];
    }
    // borders: x1 x2 y1 y2 z1 z2 at the global boundary only
    for (int a = 0; a < 3; a++) {
        m.border[2 * a] = coord[a] == 0;
        m.border[2 * a + 1] = coord[a] == parts[a] - 1;
    }
    m.fs_top = coord[2] == parts[2] - 1;
    if (m.p.pml)
        for (int a = 0; a < 3; a++)
            if ((m.border[2 * a] || (m.border[2 * a + 1] && a < 2)) && g.nPML >= n[a]) {
                err = "a part at the boundary is not thicker than the PML";
                return ST_PML_SIZE;
            }

    // padded arrays: local padded (i, j, k) is global padded (i + lo_x, ...)
    const long long np = g.npad();
    m.coord.resize(np * 3);
    m.coord_mode = -1;   // a sub-block of the global coordinates: uploaded
    m.medium.resize(np * 3);
    for (int k = 0; k < g._nz_; k++)
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const long long q = g.idx(i, j, k), Q = G.g.idx(i + lo[0], j + lo[1], k + lo[2]);
                for (int c = 0; c < 3; c++) {
                    m.coord[q * 3 + c] = G.coord[Q * 3 + c];
                    m.medium[q * 3 + c] = G.medium[Q * 3 + c];
                }
            }
    m.terrain.resize((size_t)g._nx_ * g._ny_);
    for (int j = 0; j < g._ny_; j++)
        for (int i = 0; i < g._nx_; i++)
            m.terrain[(size_t)i + (size_t)j * g._nx_] = G.terrain[(size_t)(i + lo[0]) + (size_t)(j + lo[1]) * G.g._nx_];
    // value ranges stay global (the reference reduces them over all ranks)
    m.H_min = G.H_min, m.H_max = G.H_max;
    m.Vs_min = G.Vs_min, m.Vs_max = G.Vs_max, m.Vp_min = G.Vp_min, m.Vp_max = G.Vp_max;
    m.rho_min = G.rho_min, m.rho_max = G.rho_max;
    m.dtmax = G.dtmax;
    // PML profiles: the global profiles over the part's padded range
    auto cut = [](const std::vector<float> &v, int off, int len) {
        return std::vector<float>(v.begin() + off, v.begin() + off + len);
    };
    m.pml_alpha_x = cut(G.pml_alpha_x, lo[0], g._nx_), m.pml_beta_x = cut(G.pml_beta_x, lo[0], g._nx_);
    m.pml_d_x = cut(G.pml_d_x, lo[0], g._nx_);
    m.pml_alpha_y = cut(G.pml_alpha_y, lo[1], g._ny_), m.pml_beta_y = cut(G.pml_beta_y, lo[1], g._ny_);
    m.pml_d_y = cut(G.pml_d_y, lo[1], g._ny_);
    m.pml_alpha_z = cut(G.pml_alpha_z, lo[2], g._nz_), m.pml_beta_z = cut(G.pml_beta_z, lo[2], g._nz_);
    m.pml_d_z = cut(G.pml_d_z, lo[2], g._nz_);

    auto local = [&](int I, int J, int K, int *i, int *j, int *k) {   // padded global -> padded local
        *i = I - lo[0], *j = J - lo[1], *k = K - lo[2];
        return *i >= HALO && *i < g._nx && *j >= HALO && *j < g._ny && *k >= HALO && *k < g._nz;
    };
    // finite fault: the cells of this part's interior, table rows with them
    m.fault = FaultSource();
    m.fault.nt = G.fault.nt;
    m.fault.dt = G.fault.dt;
    std::vector<long long> keep;
    for (long long c = 0; c < G.fault.npts; c++) {
        const long long Q = G.fault.index[c];
        const int I = (int)(Q % G.g._nx_), J = (int)((Q / G.g._nx_) % G.g._ny_), K = (int)(Q / ((long long)G.g._nx_ * G.g._ny_));
        int i, j, k;
        if (local(I, J, K, &i, &j, &k)) {
            keep.push_back(c);
            m.fault.index.push_back(g.idx(i, j, k));
        }
    }
    m.fault.npts = (long long)keep.size();
    m.fault.rate.resize((size_t)m.fault.npts * m.fault.nt * 6);
    for (int t = 0; t < m.fault.nt; t++)
        for (long long c = 0; c < m.fault.npts; c++)
            for (int v = 0; v < 6; v++)
                m.fault.rate[((size_t)t * m.fault.npts + c) * 6 + v] =
                    G.fault.rate[((size_t)t * G.fault.npts + keep[c]) * 6 + v];
    // point source: its 7^3 cube must lie inside one part
    m.point = G.point;
    if (G.point.kind && G.point.inside) {
        int i, j, k, cnt = 0;
        for (int dk = -3; dk <= 3; dk++)
            for (int dj = -3; dj <= 3; dj++)
                for (int di = -3; di <= 3; di++)
                    cnt += local(G.point.X + di, G.point.Y + dj, G.point.Z + dk, &i, &j, &k);
        if (cnt != 0 && cnt != 343) {
            err = "the point source's 7x7x7 smoothing cube crosses a part boundary";
            return ST_OPTIONS;
        }
        if (cnt == 343) {
            local(G.point.X, G.point.Y, G.point.Z, &i, &j, &k);
            m.point.X = i, m.point.Y = j, m.point.Z = k;
        } else {
            m.point.kind = 0;
            m.point.inside = false;
        }
    }
    // stations of this part, with their global numbers
    m.stations.clear();
    m.stations_global.clear();
    m.station_ids.clear();
    for (size_t s = 0; s < G.stations.size() / 3; s++) {
        int i, j, k;
        if (local(G.stations[s * 3], G.stations[s * 3 + 1], G.stations[s * 3 + 2], &i, &j, &k)) {
            m.stations.insert(m.stations.end(), {i, j, k});
            m.stations_global.insert(m.stations_global.end(), G.stations_global.begin() + s * 3,
                                     G.stations_global.begin() + s * 3 + 3);
            m.station_ids.push_back((int)s);
        }
    }
    return ST_OK;
}

}  // namespace cgfdm
