// Synthetic meshes and pressure-system inputs (declared in include/cfdb_synth.h).
//
// Mesh construction follows the reference mesh contract (mesh_builder.cpp:99-233): unique faces
// keyed by their sorted nodes, internal faces sorted by (owner, neighbour), boundary faces by
// (patch, owner) in first-appearance order, face nodes oriented outward from the owner. Face
// matching here uses a bucket sort on the smallest node instead of a hash map. Geometry follows
// mesh.cpp:100-186 and fv_geometry.cpp:17-69 with every vector expression evaluated in x, y, z
// order, left to right.
#include "../../include/cfdb_synth.h"
#include "../../include/cfdb.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "common.hpp"

using cfdb::fail;

namespace cfdb {
void set_thread_error(const std::string& msg); // capi.cu: the message of cfdb_last_error
} // namespace cfdb

namespace {

template <class F> int guarded_synth(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const cfdb::Error& e) {
        cfdb::set_thread_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        cfdb::set_thread_error("out of host memory");
        return CFDB_ERR_OOM;
    } catch (const std::exception& e) {
        cfdb::set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}

struct V3 {
    double x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scl(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 dvd(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// cell_shapes.hpp:22-52 (outward right-hand normals)
constexpr int kTetFaces[4][3] = {{0, 2, 1}, {0, 1, 3}, {0, 3, 2}, {1, 2, 3}};
constexpr int kHexFaces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
// 6-tet split sharing the main diagonal: permutations of the axes
constexpr int kPerms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

} // namespace

struct cfdb_mesh {
    int nx = 0, ny = 0, nz = 0;
    int n_cells = 0, n_internal = 0;
    std::vector<V3> points;
    std::vector<int> face_off{0}, face_nodes, owner, neighbour;
    std::vector<int> patch_start, patch_count;
    std::vector<V3> fc, sf, cc;
    std::vector<double> vol, delta, weights;
};

namespace {

int pid(const cfdb_mesh& m, int i, int j, int k) { return i + (m.nx + 1) * (j + (m.ny + 1) * k); }

// Patch of a boundary face from the lattice coordinates of its nodes: 2*direction + side.
int face_patch(const cfdb_mesh& m, const int* nodes, int nn) {
    int lo[3] = {1, 1, 1}, hi[3] = {1, 1, 1};
    const int n[3] = {m.nx, m.ny, m.nz};
    for (int t = 0; t < nn; ++t) {
        int p = nodes[t];
        const int i = p % (m.nx + 1);
        p /= m.nx + 1;
        const int j = p % (m.ny + 1);
        const int k = p / (m.ny + 1);
        const int c[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) {
            if (c[a] != 0) lo[a] = 0;
            if (c[a] != n[a]) hi[a] = 0;
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (lo[a]) return 2 * a;
        if (hi[a]) return 2 * a + 1;
    }
    return 6; // not on a wall: default patch
}

struct Rec {
    int key[4];
    int cell;
    int lf;
};

// MeshBuilder::build for cells of one shape (nn nodes per face, nf faces per cell).
void build(cfdb_mesh& m, const std::vector<int>& cell_nodes, int nodes_per_cell, bool tet) {
    const int nfc = tet ? 4 : 6;
    const int nn = tet ? 3 : 4;
    const int nc = m.n_cells;
    const int np = static_cast<int>(m.points.size());
    const size_t nrec = static_cast<size_t>(nc) * nfc;
    // bucket records by their smallest node
    std::vector<int> cnt(static_cast<size_t>(np) + 1, 0);
    std::vector<Rec> recs(nrec);
#pragma omp parallel for schedule(static) if (nc > 10000)
    for (int c = 0; c < nc; ++c) {
        const int* cn = cell_nodes.data() + static_cast<size_t>(c) * nodes_per_cell;
        for (int f = 0; f < nfc; ++f) {
            Rec& r = recs[static_cast<size_t>(c) * nfc + f];
            int key[4] = {-1, -1, -1, -1};
            for (int t = 0; t < nn; ++t) {
                const int v = cn[tet ? kTetFaces[f][t] : kHexFaces[f][t]];
                int u = t;
                for (; u > 0 && key[u - 1] > v; --u) key[u] = key[u - 1];
                key[u] = v;
            }
            std::memcpy(r.key, key, sizeof(key));
            r.cell = c;
            r.lf = f;
        }
    }
    for (const Rec& r : recs) ++cnt[r.key[0] + 1];
    for (int p = 0; p < np; ++p) cnt[p + 1] += cnt[p];
    std::vector<Rec> sorted(nrec);
    {
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (const Rec& r : recs) sorted[fill[r.key[0]]++] = r;
    }
    recs.clear();
    recs.shrink_to_fit();
    auto less = [](const Rec& a, const Rec& b) {
        for (int t = 1; t < 4; ++t)
            if (a.key[t] != b.key[t]) return a.key[t] < b.key[t];
        if (a.cell != b.cell) return a.cell < b.cell;
        return a.lf < b.lf;
    };
#pragma omp parallel for schedule(dynamic, 4096) if (np > 10000)
    for (int p = 0; p < np; ++p) std::sort(sorted.begin() + cnt[p], sorted.begin() + cnt[p + 1], less);
    // pair faces
    struct Face {
        int c0, lf0, c1;
    };
    std::vector<Face> internal, boundary;
    internal.reserve(nrec / 2);
    for (size_t k = 0; k < nrec;) {
        size_t e = k + 1;
        while (e < nrec && std::equal(sorted[e].key, sorted[e].key + 4, sorted[k].key)) ++e;
        if (e - k > 2) fail(CFDB_ERR_INTERNAL, "MeshBuilder: face shared by more than two cells");
        if (e - k == 2) internal.push_back({sorted[k].cell, sorted[k].lf, sorted[k + 1].cell});
        else boundary.push_back({sorted[k].cell, sorted[k].lf, -1});
        k = e;
    }
    sorted.clear();
    sorted.shrink_to_fit();
    // internal: by (owner, neighbour); owner = first cell (lower index)
    std::sort(internal.begin(), internal.end(), [](const Face& a, const Face& b) {
        return a.c0 != b.c0 ? a.c0 < b.c0 : a.c1 < b.c1;
    });
    // boundary: stable by (patch, owner) over first-appearance order (cell, local face)
    std::vector<int> bpatch(boundary.size());
    std::sort(boundary.begin(), boundary.end(), [](const Face& a, const Face& b) {
        return a.c0 != b.c0 ? a.c0 < b.c0 : a.lf0 < b.lf0;
    });
    auto face_nodes_of = [&](const Face& f, int* out) {
        const int* cn = cell_nodes.data() + static_cast<size_t>(f.c0) * nodes_per_cell;
        for (int t = 0; t < nn; ++t) out[t] = cn[tet ? kTetFaces[f.lf0][t] : kHexFaces[f.lf0][t]];
    };
    for (size_t b = 0; b < boundary.size(); ++b) {
        int nodes[4];
        face_nodes_of(boundary[b], nodes);
        bpatch[b] = face_patch(m, nodes, nn);
    }
    std::vector<size_t> border(boundary.size());
    for (size_t b = 0; b < border.size(); ++b) border[b] = b;
    std::stable_sort(border.begin(), border.end(), [&](size_t a, size_t b) {
        return bpatch[a] != bpatch[b] ? bpatch[a] < bpatch[b] : boundary[a].c0 < boundary[b].c0;
    });
    const size_t nf = internal.size() + boundary.size();
    m.n_internal = static_cast<int>(internal.size());
    m.face_off.assign(nf + 1, 0);
    m.face_nodes.resize(nf * nn);
    m.owner.resize(nf);
    m.neighbour.resize(internal.size());
    for (size_t f = 0; f < internal.size(); ++f) {
        face_nodes_of(internal[f], m.face_nodes.data() + f * nn);
        m.owner[f] = internal[f].c0;
        m.neighbour[f] = internal[f].c1;
    }
    m.patch_start.assign(7, 0);
    m.patch_count.assign(7, 0);
    for (size_t t = 0; t < border.size(); ++t) {
        const size_t f = internal.size() + t;
        const Face& bf = boundary[border[t]];
        face_nodes_of(bf, m.face_nodes.data() + f * nn);
        m.owner[f] = bf.c0;
        ++m.patch_count[bpatch[border[t]]];
    }
    int start = static_cast<int>(internal.size());
    for (int p = 0; p < 7; ++p) {
        m.patch_start[p] = start;
        start += m.patch_count[p];
    }
    for (size_t f = 0; f <= nf; ++f) m.face_off[f] = static_cast<int>(f * nn);
}

// Mesh::compute_geometry (mesh.cpp:100-186) and FvGeometry (fv_geometry.cpp:17-69).
void geometry(cfdb_mesh& m) {
    const int nf = static_cast<int>(m.owner.size());
    const int nif = m.n_internal;
    const int nc = m.n_cells;
    m.fc.resize(nf);
    m.sf.resize(nf);
#pragma omp parallel for schedule(static) if (nf > 10000)
    for (int f = 0; f < nf; ++f) {
        const int* nd = m.face_nodes.data() + m.face_off[f];
        const int np = m.face_off[f + 1] - m.face_off[f];
        if (np == 3) {
            const V3 a = m.points[nd[0]], b = m.points[nd[1]], c = m.points[nd[2]];
            m.fc[f] = dvd(add(add(a, b), c), 3.0);
            m.sf[f] = scl(cross(sub(b, a), sub(c, a)), 0.5);
            continue;
        }
        V3 pc{0.0, 0.0, 0.0};
        for (int t = 0; t < np; ++t) pc = add(pc, m.points[nd[t]]);
        pc = dvd(pc, static_cast<double>(np));
        V3 sum_n{0.0, 0.0, 0.0}, sum_ac{0.0, 0.0, 0.0};
        double sum_a = 0.0;
        for (int t = 0; t < np; ++t) {
            const V3 p0 = m.points[nd[t]], p1 = m.points[nd[(t + 1) % np]];
            const V3 n = cross(sub(p1, p0), sub(pc, p0));
            const double a = norm(n);
            sum_n = add(sum_n, n);
            sum_a += a;
            sum_ac = add(sum_ac, scl(add(add(p0, p1), pc), a));
        }
        m.fc[f] = sum_a > 1e-300 ? dvd(sum_ac, 3.0 * sum_a) : pc;
        m.sf[f] = scl(sum_n, 0.5);
    }
    std::vector<V3> est(nc, V3{0.0, 0.0, 0.0});
    std::vector<int> cnt(nc, 0);
    for (int f = 0; f < nf; ++f) {
        const int o = m.owner[f];
        est[o] = add(est[o], m.fc[f]);
        ++cnt[o];
        if (f < nif) {
            const int n = m.neighbour[f];
            est[n] = add(est[n], m.fc[f]);
            ++cnt[n];
        }
    }
    for (int c = 0; c < nc; ++c)
        if (cnt[c] > 0) est[c] = dvd(est[c], static_cast<double>(cnt[c]));
    std::vector<double> pyr(nc, 0.0);
    std::vector<V3> vc(nc, V3{0.0, 0.0, 0.0});
    for (int f = 0; f < nf; ++f) {
        const int o = m.owner[f];
        const double vo = dot(m.sf[f], sub(m.fc[f], est[o]));
        pyr[o] += vo;
        vc[o] = add(vc[o], scl(add(scl(m.fc[f], 0.75), scl(est[o], 0.25)), vo));
        if (f < nif) {
            const int n = m.neighbour[f];
            const double vn = dot(m.sf[f], sub(est[n], m.fc[f]));
            pyr[n] += vn;
            vc[n] = add(vc[n], scl(add(scl(m.fc[f], 0.75), scl(est[n], 0.25)), vn));
        }
    }
    m.vol.resize(nc);
    m.cc.resize(nc);
    for (int c = 0; c < nc; ++c) {
        m.vol[c] = pyr[c] / 3.0;
        m.cc[c] = std::fabs(pyr[c]) > 1e-300 ? dvd(vc[c], pyr[c]) : est[c];
    }
    m.delta.resize(nif);
    m.weights.resize(nif);
#pragma omp parallel for schedule(static) if (nif > 10000)
    for (int f = 0; f < nif; ++f) {
        const V3 s = m.sf[f];
        const double area = norm(s);
        const V3 cp = m.cc[m.owner[f]], cn = m.cc[m.neighbour[f]];
        const V3 d = sub(cn, cp);
        const double s_dot_d = std::max(dot(s, d), 0.05 * area * norm(d));
        m.delta[f] = area * area / s_dot_d;
        const double dp = dot(s, sub(m.fc[f], cp));
        const double dn = dot(s, sub(cn, m.fc[f]));
        const double tot = dp + dn;
        m.weights[f] = tot > 0.0 ? std::clamp(dn / tot, 0.0, 1.0) : 0.5;
    }
}

void lattice(cfdb_mesh& m, const double* xs, const double* ys, const double* zs) {
    m.points.resize(static_cast<size_t>(m.nx + 1) * (m.ny + 1) * (m.nz + 1));
    size_t t = 0;
    for (int k = 0; k <= m.nz; ++k)
        for (int j = 0; j <= m.ny; ++j)
            for (int i = 0; i <= m.nx; ++i) m.points[t++] = V3{xs[i], ys[j], zs[k]};
}

void check_lattice(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs) {
    if (nx < 1 || ny < 1 || nz < 1) fail(CFDB_ERR_BAD_ARG, "cell counts must be >= 1");
    if (!xs || !ys || !zs) fail(CFDB_ERR_BAD_ARG, "null coordinates");
    const double* ax[3] = {xs, ys, zs};
    const int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < n[a]; ++i)
            if (!(ax[a][i + 1] > ax[a][i])) fail(CFDB_ERR_BAD_ARG, "node coordinates must increase");
    if (static_cast<long long>(nx) * ny * nz * 6 >= (1LL << 31) / 4)
        fail(CFDB_ERR_BAD_ARG, "mesh too large for 32-bit face indexing");
}

} // namespace

extern "C" {

int cfdb_positions_graded(int n, double grading, double* out) {
    return guarded_synth([&] {
        if (n < 1 || out == nullptr || !(grading > 0.0)) fail(CFDB_ERR_BAD_ARG, "bad arguments");
        const double ratio = n > 1 ? std::pow(grading, 1.0 / static_cast<double>(n - 1)) : 1.0;
        for (int i = 0; i <= n; ++i) {
            out[i] = std::fabs(ratio - 1.0) < 1e-12
                         ? static_cast<double>(i) / static_cast<double>(n)
                         : (std::pow(ratio, static_cast<double>(i)) - 1.0) / (std::pow(ratio, static_cast<double>(n)) - 1.0);
        }
    });
}

int cfdb_positions_two_sided(int n, double ratio, double* out) {
    return guarded_synth([&] {
        if (n < 1 || out == nullptr || !(ratio > 0.0)) fail(CFDB_ERR_BAD_ARG, "bad arguments");
        std::vector<double> sizes(n);
        for (int i = 0; i < n; ++i) sizes[i] = std::pow(ratio, static_cast<double>(std::min(i, n - 1 - i)));
        double total = 0.0;
        for (double s : sizes) total += s;
        double acc = 0.0;
        out[0] = 0.0;
        for (int i = 0; i < n; ++i) {
            acc += sizes[i];
            out[i + 1] = acc / total;
        }
        out[n] = 1.0;
    });
}

int cfdb_mesh_box(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs, cfdb_mesh** out) {
    return guarded_synth([&] {
        check_lattice(nx, ny, nz, xs, ys, zs);
        if (out == nullptr) fail(CFDB_ERR_BAD_ARG, "null output");
        auto m = std::make_unique<cfdb_mesh>();
        m->nx = nx;
        m->ny = ny;
        m->nz = nz;
        lattice(*m, xs, ys, zs);
        m->n_cells = nx * ny * nz;
        std::vector<int> cells(static_cast<size_t>(m->n_cells) * 8);
        size_t c = 0;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const int v[8] = {pid(*m, i, j, k),         pid(*m, i + 1, j, k),         pid(*m, i + 1, j + 1, k),
                                      pid(*m, i, j + 1, k),     pid(*m, i, j, k + 1),         pid(*m, i + 1, j, k + 1),
                                      pid(*m, i + 1, j + 1, k + 1), pid(*m, i, j + 1, k + 1)};
                    std::memcpy(cells.data() + 8 * c, v, sizeof(v));
                    ++c;
                }
        build(*m, cells, 8, false);
        geometry(*m);
        *out = m.release();
    });
}

int cfdb_mesh_tet(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs, double jitter,
                  uint64_t seed, cfdb_mesh** out) {
    return guarded_synth([&] {
        check_lattice(nx, ny, nz, xs, ys, zs);
        if (out == nullptr) fail(CFDB_ERR_BAD_ARG, "null output");
        if (!(jitter >= 0.0) || jitter >= 0.25) fail(CFDB_ERR_BAD_ARG, "jitter must be in [0, 0.25)");
        auto m = std::make_unique<cfdb_mesh>();
        m->nx = nx;
        m->ny = ny;
        m->nz = nz;
        lattice(*m, xs, ys, zs);
        // jitter interior coordinates (sequential generator: reproducible)
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        const double* ax[3] = {xs, ys, zs};
        const int n[3] = {nx, ny, nz};
        size_t t = 0;
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx; ++i) {
                    const int c[3] = {i, j, k};
                    double* p = &m->points[t].x;
                    for (int a = 0; a < 3; ++a) {
                        const double r = u(rng);
                        if (c[a] == 0 || c[a] == n[a]) continue;
                        const double h = std::min(ax[a][c[a] + 1] - ax[a][c[a]], ax[a][c[a]] - ax[a][c[a] - 1]);
                        p[a] += jitter * h * r;
                    }
                    ++t;
                }
        m->n_cells = nx * ny * nz * 6;
        std::vector<int> cells(static_cast<size_t>(m->n_cells) * 4);
        size_t c = 0;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int q = 0; q < 6; ++q) {
                        int ijk[3] = {i, j, k};
                        int v[4];
                        v[0] = pid(*m, ijk[0], ijk[1], ijk[2]);
                        for (int s = 0; s < 3; ++s) {
                            ++ijk[kPerms[q][s]];
                            v[s + 1] = pid(*m, ijk[0], ijk[1], ijk[2]);
                        }
                        // odd permutations are negatively oriented on the lattice: swap 1 and 2
                        const int* pm = kPerms[q];
                        int par = 0;
                        for (int a = 0; a < 3; ++a)
                            for (int b = a + 1; b < 3; ++b)
                                if (pm[a] > pm[b]) par ^= 1;
                        if (par) std::swap(v[1], v[2]);
                        std::memcpy(cells.data() + 4 * c, v, sizeof(v));
                        ++c;
                    }
        build(*m, cells, 4, true);
        geometry(*m);
        for (int cc = 0; cc < m->n_cells; ++cc)
            if (!(m->vol[cc] > 0.0)) fail(CFDB_ERR_BAD_ARG, "jitter produced an inverted cell");
        *out = m.release();
    });
}

int cfdb_mesh_destroy(cfdb_mesh* m) {
    delete m;
    return CFDB_OK;
}

int cfdb_mesh_sizes(const cfdb_mesh* m, int* n_cells, int* n_faces, int* n_internal_faces, int* n_points) {
    if (m == nullptr) return CFDB_ERR_BAD_ARG;
    if (n_cells) *n_cells = m->n_cells;
    if (n_faces) *n_faces = static_cast<int>(m->owner.size());
    if (n_internal_faces) *n_internal_faces = m->n_internal;
    if (n_points) *n_points = static_cast<int>(m->points.size());
    return CFDB_OK;
}

int cfdb_mesh_addressing(const cfdb_mesh* m, const int** owner, const int** neighbour) {
    if (m == nullptr || owner == nullptr || neighbour == nullptr) return CFDB_ERR_BAD_ARG;
    *owner = m->owner.data();
    *neighbour = m->neighbour.data();
    return CFDB_OK;
}

int cfdb_mesh_geometry(const cfdb_mesh* m, const double** points, const double** face_centres,
                       const double** face_areas, const double** cell_centres, const double** cell_volumes) {
    if (m == nullptr) return CFDB_ERR_BAD_ARG;
    if (points) *points = &m->points[0].x;
    if (face_centres) *face_centres = &m->fc[0].x;
    if (face_areas) *face_areas = &m->sf[0].x;
    if (cell_centres) *cell_centres = &m->cc[0].x;
    if (cell_volumes) *cell_volumes = m->vol.data();
    return CFDB_OK;
}

int cfdb_mesh_faces(const cfdb_mesh* m, const int** offsets, const int** nodes) {
    if (m == nullptr || offsets == nullptr || nodes == nullptr) return CFDB_ERR_BAD_ARG;
    *offsets = m->face_off.data();
    *nodes = m->face_nodes.data();
    return CFDB_OK;
}

int cfdb_mesh_fv(const cfdb_mesh* m, const double** delta, const double** weights) {
    if (m == nullptr || delta == nullptr || weights == nullptr) return CFDB_ERR_BAD_ARG;
    *delta = m->delta.data();
    *weights = m->weights.data();
    return CFDB_OK;
}

int cfdb_synth_pressure_inputs(const cfdb_mesh* m, double sigma, int unit_rau, int flux_kind, int rhs_kind,
                               uint64_t seed, double* gamma, double* flux, double* source) {
    return guarded_synth([&] {
        if (m == nullptr || gamma == nullptr || flux == nullptr || source == nullptr)
            fail(CFDB_ERR_BAD_ARG, "null argument");
        const int nc = m->n_cells, nif = m->n_internal;
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> g01(0.0, 1.0);
        std::uniform_real_distribution<double> u11(-1.0, 1.0);
        std::vector<double> rau(nc);
        for (int c = 0; c < nc; ++c) {
            const double x = sigma > 0.0 ? std::exp(sigma * g01(rng)) : 1.0;
            rau[c] = unit_rau ? x : m->vol[c] * x;
        }
        for (int f = 0; f < nif; ++f) {
            const double w = m->weights[f];
            gamma[f] = w * rau[m->owner[f]] + (1.0 - w) * rau[m->neighbour[f]];
        }
        for (int f = 0; f < nif; ++f) {
            if (flux_kind == 0) {
                const double ux = u11(rng), uy = u11(rng), uz = u11(rng);
                flux[f] = dot(V3{ux, uy, uz}, m->sf[f]);
            } else {
                flux[f] = 0.0;
            }
        }
        if (rhs_kind == 1) {
            double mean = 0.0;
            for (int c = 0; c < nc; ++c) {
                source[c] = g01(rng);
                mean += source[c];
            }
            mean /= static_cast<double>(nc);
            for (int c = 0; c < nc; ++c) source[c] -= mean;
        } else {
            for (int c = 0; c < nc; ++c) source[c] = 0.0;
        }
    });
}

} // extern "C"
