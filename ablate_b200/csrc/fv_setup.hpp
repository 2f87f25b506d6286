// fv_setup.hpp -- host-side, one-time preparation of a rank's local mesh for the device:
// cell cones, face classes and the least-squares weights, built from the geometry DMPlex supplies.
//
// Least-squares weights restate, from the geometry alone:
//   BuildGradientReconstruction_Internal   src/finiteVolume/cellInterpolant.cpp:641-715
//     (fg->grad[side]: pseudo-inverse of each cell's neighbour offsets over its non-boundary faces)
//   LeastSquaresAverage::ComputeNeighborCellStencil  src/finiteVolume/stencils/leastSquaresAverage.cpp:71-148
//     (per-cell gradient operator over every two-sided face, used for face gradients of aux fields)
// The pseudo-inverse is computed by Householder QR of the offset matrix (full column rank), by the
// minimum-norm formula B^T (B B^T)^-1 (fewer offsets than dimensions: a boundary ghost cell), or, for
// offsets spanning fewer directions (cells next to the boundary of a tetrahedral mesh), from the
// eigen-decomposition of B^T B with the null directions dropped.
#pragma once
#include "fv_consts.hpp"
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ablate_fv.h"

namespace abl {

struct HostMesh {
    int dim = 0, n_cells = 0, n_faces = 0;
    std::vector<int32_t> face_cells;     // [nf][2]
    std::vector<uint8_t> kind;           // [nc]
    std::vector<int32_t> cone_ptr;       // [nc+1]
    std::vector<int32_t> cone_face;      // faces of each cell, by neighbour offset (canonical order)
    std::vector<int32_t> cone_nbr;       // neighbour across that face
    std::vector<uint8_t> cone_side;      // 0: the cell is the face's left cell
    std::vector<uint8_t> face_boundary;  // a boundary ghost cell is on one side
    std::vector<int32_t> flux_faces;     // faces with at least one owned cell
    std::vector<double> cgrad;           // [nf][2][3] cell-interpolant LSQ weights
    std::vector<double> fgrad;           // [nf][2][3] face-interpolant per-cell stencil weights
    std::vector<double> fdx;             // [nf][2][3] face centroid minus side-s cell centroid, in that cell's frame
};

// Pseudo-inverse through the eigen-decomposition of B^T B (cyclic Jacobi rotations), eigenvalues
// below 1e-14 of the largest treated as zero: the minimum-norm least-squares operator of a
// rank-deficient stencil (the SVD least squares PetscFVComputeGradient uses, restated).
inline void lsq_pinv_eig(int n, int dim, const double* B, double* W) {
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < n; i++)
        for (int a = 0; a < dim; a++)
            for (int b = 0; b < dim; b++) A[a][b] += B[i * dim + a] * B[i * dim + b];
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0;
        for (int a = 0; a < dim; a++)
            for (int b = a + 1; b < dim; b++) off += A[a][b] * A[a][b];
        if (off < 1e-300) break;
        for (int p = 0; p < dim; p++)
            for (int q = p + 1; q < dim; q++) {
                if (A[p][q] == 0.0) continue;
                const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < dim; k++) {  // A <- A J
                    const double x = A[k][p], y = A[k][q];
                    A[k][p] = c * x - sn * y;
                    A[k][q] = sn * x + c * y;
                }
                for (int k = 0; k < dim; k++) {  // A <- J^T A
                    const double x = A[p][k], y = A[q][k];
                    A[p][k] = c * x - sn * y;
                    A[q][k] = sn * x + c * y;
                }
                for (int k = 0; k < dim; k++) {
                    const double x = V[k][p], y = V[k][q];
                    V[k][p] = c * x - sn * y;
                    V[k][q] = sn * x + c * y;
                }
            }
    }
    double lmax = 0;
    for (int a = 0; a < dim; a++) lmax = std::max(lmax, A[a][a]);
    double Mi[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // (B^T B)^+
    for (int a = 0; a < dim; a++) {
        if (!(A[a][a] > 1e-14 * lmax)) continue;
        for (int r = 0; r < dim; r++)
            for (int s2 = 0; s2 < dim; s2++) Mi[r][s2] += V[r][a] * V[s2][a] / A[a][a];
    }
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++) {
            double acc = 0;
            for (int e = 0; e < dim; e++) acc += Mi[d][e] * B[i * dim + e];
            W[i * dim + d] = acc;
        }
}

// Pseudo-inverse of B (n x dim, row-major) returned as W (n x dim) with W[i][:] = pinv(B)[:, i].
// Full column rank: Householder QR; fewer offsets than dimensions: B^T (B B^T)^-1; a stencil whose
// offsets span fewer than min(n, dim) directions: lsq_pinv_eig.
inline void lsq_pinv(int n, int dim, const double* B, double* W) {
    if (n >= dim) {
        // numerical rank from the diagonal of R below
        bool deficient = false;
        // Householder QR: B = Q R, pinv(B) = R^-1 Q^T
        std::vector<double> A(B, B + (size_t)n * dim);  // row-major n x dim
        std::vector<double> vs((size_t)dim * n, 0.0);
        std::vector<double> beta(dim, 0.0);
        for (int j = 0; j < dim; j++) {
            double norm = 0;
            for (int i = j; i < n; i++) norm += A[i * dim + j] * A[i * dim + j];
            norm = std::sqrt(norm);
            if (norm == 0.0) {
                deficient = true;
                break;
            }
            double alpha = A[j * dim + j] > 0 ? -norm : norm;
            double* v = &vs[(size_t)j * n];
            for (int i = 0; i < n; i++) v[i] = 0;
            v[j] = A[j * dim + j] - alpha;
            for (int i = j + 1; i < n; i++) v[i] = A[i * dim + j];
            double vv = 0;
            for (int i = j; i < n; i++) vv += v[i] * v[i];
            beta[j] = vv > 0 ? 2.0 / vv : 0.0;
            for (int k = j; k < dim; k++) {
                double s = 0;
                for (int i = j; i < n; i++) s += v[i] * A[i * dim + k];
                s *= beta[j];
                for (int i = j; i < n; i++) A[i * dim + k] -= s * v[i];
            }
        }
        double rmax = 0;
        if (!deficient)
            for (int j = 0; j < dim; j++) rmax = std::max(rmax, std::fabs(A[j * dim + j]));
        if (!deficient)
            for (int j = 0; j < dim; j++)
                if (!(std::fabs(A[j * dim + j]) > 1e-7 * rmax)) deficient = true;
        if (deficient) {
            lsq_pinv_eig(n, dim, B, W);
            return;
        }
        // columns of pinv: solve R x = (Q^T e_i)[0:dim] for each i
        std::vector<double> q(n);
        for (int i = 0; i < n; i++) {
            for (int r = 0; r < n; r++) q[r] = (r == i) ? 1.0 : 0.0;
            for (int j = 0; j < dim; j++) {
                const double* v = &vs[(size_t)j * n];
                double s = 0;
                for (int r = j; r < n; r++) s += v[r] * q[r];
                s *= beta[j];
                for (int r = j; r < n; r++) q[r] -= s * v[r];
            }
            double x[3];
            for (int j = dim - 1; j >= 0; j--) {
                double s = q[j];
                for (int k = j + 1; k < dim; k++) s -= A[j * dim + k] * x[k];
                x[j] = s / A[j * dim + j];
            }
            for (int j = 0; j < dim; j++) W[i * dim + j] = x[j];
        }
    } else {
        // minimum norm: pinv(B) = B^T (B B^T)^-1, n < dim (n = 1 or 2)
        double G[2][2] = {{0, 0}, {0, 0}};
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++)
                for (int d = 0; d < dim; d++) G[a][b] += B[a * dim + d] * B[b * dim + d];
        double Gi[2][2];
        if (n == 1) {
            Gi[0][0] = 1.0 / G[0][0];
        } else {
            double det = G[0][0] * G[1][1] - G[0][1] * G[1][0];
            if (!(std::fabs(det) > 1e-14 * G[0][0] * G[1][1])) {  // parallel offsets
                lsq_pinv_eig(n, dim, B, W);
                return;
            }
            Gi[0][0] = G[1][1] / det;
            Gi[1][1] = G[0][0] / det;
            Gi[0][1] = -G[0][1] / det;
            Gi[1][0] = -G[1][0] / det;
        }
        for (int i = 0; i < n; i++)
            for (int d = 0; d < dim; d++) {
                double s = 0;
                for (int a = 0; a < n; a++) s += B[a * dim + d] * Gi[a][i];
                W[i * dim + d] = s;
            }
    }
}

// Cell tiles for the fused flux kernel: owned cells sorted along a Morton curve of their centroids
// and cut into runs of at most `tile_cells` cells (on power-of-two boxes each run is a compact block).
// Every tile lists all flux faces of its cells (faces shared by two tiles appear in both lists), with
// the face geometry copied into tile order so the kernel streams it, and for every tile cell the
// (local face, side) pairs in ascending global face order.
//
// The face records of a tile are in ascending face order. For the adjoint they are also coloured so
// that no two faces of one colour touch the same tile cell, and listed colour by colour (tf_adj,
// col_start). The adjoint kernel accumulates per-cell sums in shared memory one colour at a time,
// which needs no atomics and fixes the summation order. A face with a side that is not an owned cell (a boundary ghost or a partition
// halo) is in exactly one tile; its contribution to that side goes to a per-face record (nb index).
struct Tiles {
    int n_tiles = 0;
    int max_faces = 0;                    // largest per-tile face count (sizes shared memory)
    std::vector<int32_t> cell_ptr;        // [n_tiles+1] into cells
    std::vector<int32_t> cells;           // owned cells grouped by tile
    std::vector<int32_t> face_ptr;        // [n_tiles+1] into the tile-face records
    std::vector<int32_t> tf_cells;        // [ntf][2] global left/right cell
    std::vector<int32_t> tf_face;         // [ntf] global face
    std::vector<double> tf_normal;        // [ntf][3]
    std::vector<double> tf_fdx;           // [ntf][6] face centroid minus each side's centroid
    std::vector<int32_t> tc_fptr;         // [n_owned+1] per tile cell into tc_face
    std::vector<uint16_t> tc_face;        // local face index | side << 15
    std::vector<uint32_t> tf_slot;        // [ntf] tile-local slot of L | of R << 16 (0xffff: not a tile cell)
    std::vector<uint16_t> tf_adj;         // [ntf] per tile, the record of its k-th face in adjoint colour order
    std::vector<int32_t> tf_nb;           // [ntf] record of the non-owned side, -1 if both sides are owned
    std::vector<int32_t> col_base;        // [n_tiles+1] into col_start
    std::vector<int32_t> col_start;       // per tile: first position (in tf_adj) of each adjoint colour, then the end
    std::vector<int32_t> face_nb;         // [n_faces] record index of faces with a non-owned side, else -1
    int n_nb = 0;                         // number of such records
    int max_colors = 0;
};

inline uint64_t morton_spread(uint64_t x, int dim) {
    if (dim == 1) return x;
    uint64_t r = 0;
    for (int b = 0; b < (dim == 2 ? 31 : 21); b++) r |= ((x >> b) & 1ull) << (b * dim);
    return r;
}

// morton = false keeps the caller's own cell order (compact when the DM was permuted along a
// space-filling curve); true sorts owned cells by the Morton code of their centroids.
inline Tiles build_tiles(const HostMesh& h, const abl_mesh_desc* m, int tile_cells, bool morton = true) {
    Tiles t;
    const int dim = h.dim;
    std::vector<int32_t> owned;
    for (int c = 0; c < h.n_cells; c++)
        if (h.kind[c] == ABL_CELL_OWNED) owned.push_back(c);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c : owned)
        for (int d = 0; d < dim; d++) {
            lo[d] = std::min(lo[d], m->cell_centroid[3 * (size_t)c + d]);
            hi[d] = std::max(hi[d], m->cell_centroid[3 * (size_t)c + d]);
        }
    const int bits = dim == 1 ? 62 : (dim == 2 ? 31 : 21);
    (void)bits;
    const double scale = std::ldexp(1.0, bits) - 1.0;
    std::vector<std::pair<uint64_t, int32_t>> keyed(owned.size());
    for (size_t i = 0; i < owned.size(); i++) {
        const int c = owned[i];
        uint64_t key = 0;
        for (int d = 0; d < dim; d++) {
            const double span = hi[d] - lo[d];
            const double u = span > 0 ? (m->cell_centroid[3 * (size_t)c + d] - lo[d]) / span : 0.0;
            key |= morton_spread((uint64_t)(u * scale), dim) << d;
        }
        keyed[i] = {morton ? key : (uint64_t)i, c};
    }
    std::sort(keyed.begin(), keyed.end());
    const int n = (int)keyed.size();
    t.n_tiles = (n + tile_cells - 1) / tile_cells;
    t.cell_ptr.resize(t.n_tiles + 1);
    t.cells.resize(n);
    for (int i = 0; i < n; i++) t.cells[i] = keyed[i].second;
    for (int k = 0; k <= t.n_tiles; k++) t.cell_ptr[k] = std::min(n, k * tile_cells);
    std::vector<int32_t> local(h.n_cells, -1);
    std::vector<int32_t> faces;
    t.face_ptr.push_back(0);
    t.tc_fptr.assign(n + 1, 0);
    t.col_base.push_back(0);
    std::vector<std::vector<uint16_t>> lists;
    t.face_nb.assign(h.n_faces, -1);
    for (int f : h.flux_faces)
        if (h.kind[h.face_cells[2 * f]] != ABL_CELL_OWNED || h.kind[h.face_cells[2 * f + 1]] != ABL_CELL_OWNED) t.face_nb[f] = t.n_nb++;
    for (int k = 0; k < t.n_tiles; k++) {
        const int cb = t.cell_ptr[k], ce = t.cell_ptr[k + 1];
        faces.clear();
        for (int j = cb; j < ce; j++) {
            const int c = t.cells[j];
            local[c] = j - cb;
            for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) faces.push_back(h.cone_face[i]);
        }
        std::sort(faces.begin(), faces.end());
        faces.erase(std::unique(faces.begin(), faces.end()), faces.end());
        if (faces.size() > 0x7fff) throw std::invalid_argument("tile has too many faces");
        t.max_faces = std::max(t.max_faces, (int)faces.size());
        lists.assign(ce - cb, {});
        // face records in global face order (the flux pass reads them in this order, neighbouring
        // threads on neighbouring faces: the fastest of the orders measured)
        const int base = (int)(t.tf_cells.size() / 2);
        for (size_t i = 0; i < faces.size(); i++) {
            const int f = faces[i];
            const int L = h.face_cells[2 * f], R = h.face_cells[2 * f + 1];
            t.tf_cells.push_back(L);
            t.tf_cells.push_back(R);
            t.tf_face.push_back(f);
            for (int d = 0; d < 3; d++) t.tf_normal.push_back(d < dim ? m->face_normal[3 * (size_t)f + d] : 0.0);
            for (int z = 0; z < 6; z++) t.tf_fdx.push_back(h.fdx[6 * (size_t)f + z]);
            t.tf_slot.push_back((uint32_t)(local[L] >= 0 ? local[L] : 0xffff) | ((uint32_t)(local[R] >= 0 ? local[R] : 0xffff) << 16));
            t.tf_nb.push_back(t.face_nb[f]);
        }
        // the adjoint's colouring: balanced greedy. With K colours allowed each face takes the
        // least-filled colour free at both its cells; K starts at the bound ceil(faces / kColorCap) and
        // grows until every face fits. On an 8x8x4 hex tile (896 faces) that is 8 passes of 112 faces
        // where first-fit needs 12 (six of them part-empty), and every pass ends at a CTA barrier.
        std::vector<int> bcol;
        int nb_col = 0;
        for (int K = std::max(1, ((int)faces.size() + kColorCap - 1) / kColorCap); K <= 64 && nb_col == 0; K++) {
            std::vector<uint64_t> u2(ce - cb, 0);
            std::vector<int> c2(K, 0);
            bcol.assign(faces.size(), 0);
            bool fits = true;
            for (size_t i = 0; i < faces.size() && fits; i++) {
                const int f = faces[i];
                const int lL = local[h.face_cells[2 * f]], lR = local[h.face_cells[2 * f + 1]];
                const uint64_t busy = (lL >= 0 ? u2[lL] : 0) | (lR >= 0 ? u2[lR] : 0);
                int c = -1;
                for (int k = 0; k < K; k++)
                    if (!((busy >> k) & 1ull) && c2[k] < kColorCap && (c < 0 || c2[k] < c2[c])) c = k;
                if (c < 0) fits = false;
                else {
                    bcol[i] = c;
                    c2[c]++;
                    if (lL >= 0) u2[lL] |= 1ull << c;
                    if (lR >= 0) u2[lR] |= 1ull << c;
                }
            }
            if (fits) nb_col = K;
        }
        if (nb_col == 0) throw std::invalid_argument("tile face colouring needs more than 64 colours");
        t.max_colors = std::max(t.max_colors, nb_col);
        std::vector<int> aorder(faces.size());
        for (size_t i = 0; i < faces.size(); i++) aorder[i] = (int)i;
        std::stable_sort(aorder.begin(), aorder.end(), [&](int a, int b) { return bcol[a] < bcol[b]; });
        for (size_t q = 0; q < aorder.size(); q++) {
            if (q == 0 || bcol[aorder[q - 1]] != bcol[aorder[q]]) t.col_start.push_back(base + (int)q);
            t.tf_adj.push_back((uint16_t)aorder[q]);
        }
        t.col_start.push_back(base + (int)faces.size());
        t.col_base.push_back((int)t.col_start.size());
        // per-cell lists in ascending global face order, pointing at the face records
        for (size_t i = 0; i < faces.size(); i++) {
            const int f = faces[i];
            const int L = h.face_cells[2 * f], R = h.face_cells[2 * f + 1];
            if (local[L] >= 0) lists[local[L]].push_back((uint16_t)i);
            if (local[R] >= 0) lists[local[R]].push_back((uint16_t)(i | 0x8000));
        }
        for (int j = cb; j < ce; j++) {
            t.tc_fptr[j + 1] = t.tc_fptr[j] + (int)lists[j - cb].size();
            t.tc_face.insert(t.tc_face.end(), lists[j - cb].begin(), lists[j - cb].end());
            local[t.cells[j]] = -1;
        }
        t.face_ptr.push_back((int32_t)(t.tf_cells.size() / 2));
    }
    return t;
}

inline HostMesh build_host_mesh(const abl_mesh_desc* m, bool need_cgrad, bool need_fgrad) {
    HostMesh h;
    if (!m || m->dim < 1 || m->dim > 3 || m->n_cells <= 0 || m->n_faces < 0 || !m->face_cells || !m->face_normal || !m->face_centroid ||
        !m->cell_centroid || !m->cell_volume)
        throw std::invalid_argument("invalid mesh descriptor");
    h.dim = m->dim;
    h.n_cells = m->n_cells;
    h.n_faces = m->n_faces;
    const int nc = h.n_cells, nf = h.n_faces, dim = h.dim;
    h.face_cells.assign(m->face_cells, m->face_cells + 2 * (size_t)nf);
    h.kind.assign(nc, ABL_CELL_OWNED);
    if (m->cell_kind)
        for (int c = 0; c < nc; c++) {
            if (m->cell_kind[c] > ABL_CELL_HALO_OUTER) throw std::invalid_argument("invalid cell kind");
            h.kind[c] = m->cell_kind[c];
        }
    for (int c = 0; c < nc; c++)
        if (!(m->cell_volume[c] > 0.0)) throw std::invalid_argument("cell volume must be positive (cell " + std::to_string(c) + ")");
    h.cone_ptr.assign(nc + 1, 0);
    for (int f = 0; f < nf; f++) {
        int a = h.face_cells[2 * f], b = h.face_cells[2 * f + 1];
        if (a < 0 || a >= nc || b < 0 || b >= nc || a == b) throw std::invalid_argument("face " + std::to_string(f) + " has an invalid support");
        h.cone_ptr[a + 1]++;
        h.cone_ptr[b + 1]++;
    }
    for (int c = 0; c < nc; c++) h.cone_ptr[c + 1] += h.cone_ptr[c];
    const size_t ncone = h.cone_ptr[nc];
    h.cone_face.resize(ncone);
    h.cone_nbr.resize(ncone);
    h.cone_side.resize(ncone);
    std::vector<int32_t> fill(h.cone_ptr.begin(), h.cone_ptr.end() - 1);
    for (int f = 0; f < nf; f++)
        for (int s = 0; s < 2; s++) {
            int c = h.face_cells[2 * f + s];
            int i = fill[c]++;
            h.cone_face[i] = f;
            h.cone_nbr[i] = h.face_cells[2 * f + (1 - s)];
            h.cone_side[i] = (uint8_t)s;
        }
    for (int c = 0; c < nc; c++)
        if (h.kind[c] == ABL_CELL_BOUNDARY && h.cone_ptr[c + 1] - h.cone_ptr[c] != 1)
            throw std::invalid_argument("boundary ghost cell " + std::to_string(c) + " must have exactly one face");
    h.face_boundary.assign(nf, 0);
    for (int f = 0; f < nf; f++) {
        uint8_t ka = h.kind[h.face_cells[2 * f]], kb = h.kind[h.face_cells[2 * f + 1]];
        h.face_boundary[f] = (ka == ABL_CELL_BOUNDARY || kb == ABL_CELL_BOUNDARY);
        if (ka == ABL_CELL_OWNED || kb == ABL_CELL_OWNED) h.flux_faces.push_back(f);
    }
    // offset from each side's cell centroid to the face centroid, periodic images resolved
    h.fdx.assign((size_t)nf * 6, 0.0);
    for (int f = 0; f < nf; f++) {
        const int a = h.face_cells[2 * f], b = h.face_cells[2 * f + 1];
        for (int d = 0; d < dim; d++) {
            const double sh = m->face_shift ? m->face_shift[3 * (size_t)f + d] : 0.0;
            h.fdx[6 * (size_t)f + d] = m->face_centroid[3 * (size_t)f + d] - m->cell_centroid[3 * (size_t)a + d];
            h.fdx[6 * (size_t)f + 3 + d] = (m->face_centroid[3 * (size_t)f + d] - sh) - m->cell_centroid[3 * (size_t)b + d];
        }
    }
    // neighbour offset x_n - x_c across cone entry i (periodic images resolved)
    auto nbr_dx = [&](int c, int i, int d) {
        const int f = h.cone_face[i];
        const int n = h.cone_nbr[i];
        const double sh = m->face_shift ? m->face_shift[3 * (size_t)f + d] : 0.0;
        const double xn = m->cell_centroid[3 * (size_t)n + d] + (h.cone_side[i] == 0 ? sh : -sh);
        return xn - m->cell_centroid[3 * (size_t)c + d];
    };
    // each cell's cone in one canonical order: by the neighbour offset x_n - x_c (lexicographic), then
    // by face index. The cells of a structured block then list their neighbours alike and get bitwise
    // the same least-squares weights, and cone entry i points the same way for neighbouring cells.
    {
        std::vector<std::pair<std::array<double, 3>, int>> key;
        std::vector<int32_t> cf, cn;
        std::vector<uint8_t> cs;
        for (int c = 0; c < nc; c++) {
            const int b = h.cone_ptr[c], n = h.cone_ptr[c + 1] - b;
            if (n < 2) continue;
            key.clear();
            for (int i = b; i < b + n; i++) {
                std::array<double, 3> v{0.0, 0.0, 0.0};
                for (int d = 0; d < dim; d++) v[d] = nbr_dx(c, i, d);
                key.push_back({v, i});
            }
            std::sort(key.begin(), key.end(), [&](const auto& x, const auto& y) {
                if (x.first != y.first) return x.first < y.first;
                return h.cone_face[x.second] < h.cone_face[y.second];
            });
            cf.resize(n);
            cn.resize(n);
            cs.resize(n);
            for (int k = 0; k < n; k++) {
                cf[k] = h.cone_face[key[k].second];
                cn[k] = h.cone_nbr[key[k].second];
                cs[k] = h.cone_side[key[k].second];
            }
            std::copy(cf.begin(), cf.end(), h.cone_face.begin() + b);
            std::copy(cn.begin(), cn.end(), h.cone_nbr.begin() + b);
            std::copy(cs.begin(), cs.end(), h.cone_side.begin() + b);
        }
    }
    std::vector<double> B, W;
    if (need_cgrad) {
        h.cgrad.assign((size_t)nf * 6, 0.0);
        for (int c = 0; c < nc; c++) {
            if (h.kind[c] != ABL_CELL_OWNED && h.kind[c] != ABL_CELL_HALO) continue;
            B.clear();
            std::vector<size_t> slots;
            for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
                if (h.face_boundary[h.cone_face[i]]) continue;
                for (int d = 0; d < dim; d++) B.push_back(nbr_dx(c, i, d));
                slots.push_back((size_t)h.cone_face[i] * 6 + 3 * h.cone_side[i]);
            }
            if (slots.empty()) throw std::invalid_argument("isolated cell " + std::to_string(c) + " has no neighbours");
            W.assign(B.size(), 0.0);
            lsq_pinv((int)slots.size(), dim, B.data(), W.data());
            for (size_t i = 0; i < slots.size(); i++)
                for (int d = 0; d < dim; d++) h.cgrad[slots[i] + d] = W[i * dim + d];
        }
    }
    if (need_fgrad) {
        h.fgrad.assign((size_t)nf * 6, 0.0);
        for (int c = 0; c < nc; c++) {
            if (h.kind[c] == ABL_CELL_HALO_OUTER) continue;
            B.clear();
            std::vector<size_t> slots;
            for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
                for (int d = 0; d < dim; d++) B.push_back(nbr_dx(c, i, d));
                slots.push_back((size_t)h.cone_face[i] * 6 + 3 * h.cone_side[i]);
            }
            if (slots.empty()) continue;
            W.assign(B.size(), 0.0);
            lsq_pinv((int)slots.size(), dim, B.data(), W.data());
            for (size_t i = 0; i < slots.size(); i++)
                for (int d = 0; d < dim; d++) h.fgrad[slots[i] + d] = W[i * dim + d];
        }
    }
    return h;
}

// Classes of n items that are equal bit for bit: hash(k) gives item k's hash, same(a, b) compares two
// items. Fills cls[k] with item k's class (classes numbered in order of first appearance) and rep[j]
// with the first item of class j, and returns the number of classes; returns 0 as soon as there are
// more than max_cls.
template <class Hash, class Same>
inline size_t distinct_classes(size_t n, size_t max_cls, Hash hash, Same same, std::vector<int32_t>& cls, std::vector<size_t>& rep) {
    std::unordered_multimap<uint64_t, int32_t> seen;
    cls.assign(n, -1);
    rep.clear();
    for (size_t k = 0; k < n; k++) {
        const uint64_t hk = hash(k);
        const auto range = seen.equal_range(hk);
        for (auto it = range.first; it != range.second; ++it)
            if (same(rep[(size_t)it->second], k)) {
                cls[k] = it->second;
                break;
            }
        if (cls[k] >= 0) continue;
        if (rep.size() == max_cls) return 0;
        cls[k] = (int32_t)rep.size();
        seen.emplace(hk, cls[k]);
        rep.push_back(k);
    }
    return rep.size();
}

// a hash of the bits of n doubles, continuing from h: per word, xor, multiply by the 64-bit FNV prime
// and fold the high bits down
inline uint64_t hash_bits(const double* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for (size_t i = 0; i < n; i++) {
        uint64_t b;
        std::memcpy(&b, p + i, sizeof b);
        h = (h ^ b) * 1099511628211ull;
        h ^= h >> 29;
    }
    return h;
}

// Record tables are used when the distinct records are at most this many and at most 1/8 of the items.
constexpr size_t kMaxRecordClasses = 4096;

// Per cone entry (cell-major, the cone in its canonical order): the LSQ state weight (0 across a
// boundary face and without a state gradient) and the aux weight packed in one 6-double record (cwa),
// the neighbour offset x_n - x_c (cv), and the neighbour's two weights for the same face packed like
// cwa (cwar: the transposed operators of the adjoint gather). With tables, cells whose sequences (cwa,
// cv, cwar over the cone) are equal bit for bit share one copy: the arrays then hold one sequence per
// class and base[c] is the first entry of cell c's copy.
struct ConeRecords {
    std::vector<double> cwa, cv, cwar;
    std::vector<int32_t> base;  // empty: one record per cone entry
    size_t classes = 0;
    int max_cone = 0;
};

inline ConeRecords cone_records(const HostMesh& h, bool lsq, bool dif, bool tables) {
    ConeRecords r;
    const size_t ncone = h.cone_face.size();
    r.cwa.assign(6 * ncone, 0.0);
    r.cv.assign(3 * ncone, 0.0);
    r.cwar.assign(6 * ncone, 0.0);
    for (int c = 0; c < h.n_cells; c++) {
        r.max_cone = std::max(r.max_cone, h.cone_ptr[c + 1] - h.cone_ptr[c]);
        for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
            const size_t f = (size_t)h.cone_face[i], sc = h.cone_side[i], q = (size_t)i;
            for (int d = 0; d < 3; d++) {
                if (lsq && !h.face_boundary[f]) {
                    r.cwa[6 * q + d] = h.cgrad[6 * f + 3 * sc + d];
                    r.cwar[6 * q + d] = h.cgrad[6 * f + 3 * (1 - sc) + d];
                }
                if (dif) {
                    r.cwa[6 * q + 3 + d] = h.fgrad[6 * f + 3 * sc + d];
                    r.cwar[6 * q + 3 + d] = h.fgrad[6 * f + 3 * (1 - sc) + d];
                }
                r.cv[3 * q + d] = h.fdx[6 * f + 3 * sc + d] - h.fdx[6 * f + 3 * (1 - sc) + d];
            }
        }
    }
    if (!tables || h.n_cells < 8) return r;
    auto span = [&](size_t c) { return std::make_pair((size_t)h.cone_ptr[c], (size_t)(h.cone_ptr[c + 1] - h.cone_ptr[c])); };
    auto seq_hash = [&](size_t c) {
        const auto [b, n] = span(c);
        uint64_t hh = hash_bits(&r.cwa[6 * b], 6 * n);
        hh = hash_bits(&r.cv[3 * b], 3 * n, hh);
        return hash_bits(&r.cwar[6 * b], 6 * n, hh);
    };
    auto seq_same = [&](size_t a, size_t c) {
        const auto [ba, na] = span(a);
        const auto [bc, nn] = span(c);
        return na == nn && std::memcmp(&r.cwa[6 * ba], &r.cwa[6 * bc], 6 * nn * sizeof(double)) == 0 &&
               std::memcmp(&r.cv[3 * ba], &r.cv[3 * bc], 3 * nn * sizeof(double)) == 0 &&
               std::memcmp(&r.cwar[6 * ba], &r.cwar[6 * bc], 6 * nn * sizeof(double)) == 0;
    };
    std::vector<int32_t> cls;
    std::vector<size_t> rep;
    const size_t ncl = distinct_classes((size_t)h.n_cells, std::min(kMaxRecordClasses, (size_t)h.n_cells / 8), seq_hash, seq_same, cls, rep);
    if (!ncl) return r;
    std::vector<int32_t> start(ncl + 1, 0);
    for (size_t j = 0; j < ncl; j++) start[j + 1] = start[j] + (int32_t)span(rep[j]).second;
    const size_t nt = (size_t)start[ncl];
    std::vector<double> tw(6 * nt), tv(3 * nt), twr(6 * nt);
    for (size_t j = 0; j < ncl; j++) {
        const auto [b, n] = span(rep[j]);
        const size_t o = (size_t)start[j];
        std::copy_n(&r.cwa[6 * b], 6 * n, &tw[6 * o]);
        std::copy_n(&r.cv[3 * b], 3 * n, &tv[3 * o]);
        std::copy_n(&r.cwar[6 * b], 6 * n, &twr[6 * o]);
    }
    r.base.resize(h.n_cells);
    for (int c = 0; c < h.n_cells; c++) r.base[c] = start[cls[c]];
    r.cwa.swap(tw);
    r.cv.swap(tv);
    r.cwar.swap(twr);
    r.classes = ncl;
    return r;
}

// Per tile face record one 10-double geometry record: area normal (3), the face centroid minus each
// side's centroid (6), a pad. With tables, records equal bit for bit are stored once and cls[i] gives
// record i's copy.
struct GeoRecords {
    std::vector<double> geo;
    std::vector<uint16_t> cls;  // empty: one record per tile face record
};

inline GeoRecords tile_geometry(const Tiles& tl, bool tables) {
    GeoRecords g;
    const size_t ntf = tl.tf_cells.size() / 2;
    g.geo.assign(10 * ntf, 0.0);
    for (size_t i = 0; i < ntf; i++) {
        for (int d = 0; d < 3; d++) g.geo[10 * i + d] = tl.tf_normal[3 * i + d];
        for (int z = 0; z < 6; z++) g.geo[10 * i + 3 + z] = tl.tf_fdx[6 * i + z];
    }
    if (!tables || ntf < 8) return g;
    std::vector<int32_t> cls;
    std::vector<size_t> rep;
    const size_t ng = distinct_classes(
        ntf, std::min(kMaxRecordClasses, ntf / 8), [&](size_t k) { return hash_bits(&g.geo[10 * k], 10); },
        [&](size_t a, size_t b) { return std::memcmp(&g.geo[10 * a], &g.geo[10 * b], 10 * sizeof(double)) == 0; }, cls, rep);
    if (!ng) return g;
    std::vector<double> table(10 * ng);
    for (size_t j = 0; j < ng; j++) std::copy_n(&g.geo[10 * rep[j]], 10, &table[10 * j]);
    g.geo.swap(table);
    g.cls.assign(cls.begin(), cls.end());
    return g;
}

// Order in which a cell sums its faces in the fused kernel: its cone (canonical, by neighbour offset)
// sorted by the axis of the offset's largest component, then its sign. On a hex cell that is x-, x+,
// y-, y+, z-, z+: opposite faces are summed next to each other, so equal and opposite fluxes cancel
// exactly (a uniform state keeps a zero residual). The order depends on the cell's geometry alone, so it
// is the same in every tile and every partition.
inline int face_sum_key(const HostMesh& h, int i) {
    const size_t f = (size_t)h.cone_face[i];
    const int s = h.cone_side[i];
    int axis = 0;
    double best = -1.0, v = 0.0;
    for (int d = 0; d < h.dim; d++) {
        const double x = h.fdx[6 * f + 3 * s + d] - h.fdx[6 * f + 3 * (1 - s) + d];  // x_n - x_c
        if (std::fabs(x) > best) {
            best = std::fabs(x);
            axis = d;
            v = x;
        }
    }
    return 2 * axis + (v > 0 ? 1 : 0);
}

// Tables of the fused one-pass RHS (k_fused_rhs). Per tile its ext cells: the tile's cells (in tile
// order), then ring 1 (the cells across the tile's faces), then ring 2 (the further neighbours of
// ring 1), each ring in the order a walk of the previous one meets them (cells in order, each cone in
// its canonical order). The tile's faces are listed in the order a walk of its cells' cones meets
// them, and every tile cell lists its faces in face_sum_key order. All of it follows from the local
// geometry, so the tiles of a structured block get equal tables; the local topology of a tile (cones,
// faces, face lists in local slots, kinds, weight and geometry records) is one run of int words, and
// tiles whose runs are equal word for word share one copy (class).
struct FusedTiles {
    int max_ext = 0, max_grad = 0, max_faces = 0;
    std::vector<int32_t> ext_ptr;   // [n_tiles + 1]
    std::vector<int32_t> ext;       // global cell per ext slot
    std::vector<int32_t> tile_cls;  // [n_tiles]
    std::vector<int32_t> cls_off;   // [n_classes] into pool
    std::vector<int32_t> pool;
};

// weight_base[c]: first weight record of cell c's cone (its class copy, or its own cone start);
// geo_cls: per tile face record its geometry record (empty: the record index itself)
inline FusedTiles fused_tiles(const HostMesh& h, const Tiles& tl, const std::vector<int32_t>& weight_base, const std::vector<uint16_t>& geo_cls) {
    FusedTiles ft;
    std::vector<int32_t> slot(h.n_cells, -1), fidx(h.n_faces, -1), rec_of(h.n_faces, -1);
    std::vector<int32_t> ext, words, flist;
    std::vector<std::pair<int, int>> order;
    std::unordered_multimap<uint64_t, int32_t> seen;
    ft.ext_ptr.push_back(0);
    for (int k = 0; k < tl.n_tiles; k++) {
        const int cb = tl.cell_ptr[k], ce = tl.cell_ptr[k + 1], nt = ce - cb;
        ext.clear();
        for (int j = cb; j < ce; j++) {
            slot[tl.cells[j]] = (int32_t)ext.size();
            ext.push_back(tl.cells[j]);
        }
        // ring 1, then ring 2
        size_t from = 0;
        int ng = 0;
        for (int ring = 0; ring < 2; ring++) {
            const size_t to = ext.size();
            for (size_t q = from; q < to; q++) {
                const int c = ext[q];
                for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
                    const int n = h.cone_nbr[i];
                    if (slot[n] < 0) {
                        slot[n] = (int32_t)ext.size();
                        ext.push_back(n);
                    }
                }
            }
            if (ring == 0) ng = (int)ext.size();
            from = to;
        }
        const int ne = (int)ext.size();
        if (ne > 0xffff) throw std::invalid_argument("fused tile has too many ext cells");
        // the tile's faces in walk order, and each face's record among the tile's face records
        flist.clear();
        for (int j = 0; j < nt; j++)
            for (int i = h.cone_ptr[ext[j]]; i < h.cone_ptr[ext[j] + 1]; i++) {
                const int f = h.cone_face[i];
                if (fidx[f] < 0) {
                    fidx[f] = (int32_t)flist.size();
                    flist.push_back(f);
                }
            }
        const int fb = tl.face_ptr[k], fe = tl.face_ptr[k + 1], nf = (int)flist.size();
        if (nf != fe - fb || nf > 0x7fff) throw std::logic_error("fused tile faces differ from the tile's face records");
        for (int i = fb; i < fe; i++) rec_of[tl.tf_face[i]] = i;
        words.assign({nt, ng, ne, nf});
        // cone starts, weight bases, kinds, neighbour slots
        int acc = 0;
        for (int j = 0; j < ng; j++) {
            words.push_back(acc);
            acc += h.cone_ptr[ext[j] + 1] - h.cone_ptr[ext[j]];
        }
        words.push_back(acc);
        for (int j = 0; j < ng; j++) words.push_back(weight_base[ext[j]]);
        for (int j = 0; j < ng; j++) words.push_back(h.kind[ext[j]]);
        for (int j = 0; j < ng; j++) {
            const int c = ext[j];
            for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++)
                words.push_back(slot[h.cone_nbr[i]] | (h.face_boundary[h.cone_face[i]] ? (1 << 16) : 0));
        }
        for (int f : flist) {
            const int L = h.face_cells[2 * (size_t)f], R = h.face_cells[2 * (size_t)f + 1];
            if (slot[L] < 0 || slot[L] >= ng || slot[R] < 0 || slot[R] >= ng) throw std::logic_error("fused tile face outside ring 1");
            words.push_back(slot[L] | (slot[R] << 16));
        }
        for (int f : flist) {
            if (rec_of[f] < 0) throw std::logic_error("fused tile face without a record");
            words.push_back(geo_cls.empty() ? rec_of[f] : (int32_t)geo_cls[rec_of[f]]);
        }
        // per tile cell its faces in face_sum_key order: local face | side << 15 (side 1: the cell is the
        // face's right cell and adds the flux)
        const size_t tcp0 = words.size();
        words.resize(words.size() + nt + 1);
        int ntc = 0;
        std::vector<int32_t> entries;
        for (int j = 0; j < nt; j++) {
            const int c = ext[j];
            order.clear();
            for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) order.push_back({face_sum_key(h, i), i});
            std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            words[tcp0 + j] = ntc;
            for (const auto& o : order) {
                entries.push_back(fidx[h.cone_face[o.second]] | (h.cone_side[o.second] ? 0x8000 : 0));
                ntc++;
            }
        }
        words[tcp0 + nt] = ntc;
        words.insert(words.end(), entries.begin(), entries.end());
        for (int f : flist) {
            fidx[f] = -1;
            rec_of[f] = -1;
        }
        for (int i = fb; i < fe; i++) rec_of[tl.tf_face[i]] = -1;
        for (int c : ext) slot[c] = -1;
        ft.ext.insert(ft.ext.end(), ext.begin(), ext.end());
        ft.ext_ptr.push_back((int32_t)ft.ext.size());
        ft.max_ext = std::max(ft.max_ext, ne);
        ft.max_grad = std::max(ft.max_grad, ng);
        ft.max_faces = std::max(ft.max_faces, nf);
        // one copy per distinct run of words
        uint64_t hk = 1469598103934665603ull;
        for (int32_t x : words) {
            hk = (hk ^ (uint32_t)x) * 1099511628211ull;
            hk ^= hk >> 29;
        }
        int32_t cls = -1;
        const auto range = seen.equal_range(hk);
        for (auto it = range.first; it != range.second && cls < 0; ++it) {
            const int32_t o = ft.cls_off[it->second];
            const size_t len = (it->second + 1 < (int32_t)ft.cls_off.size() ? (size_t)ft.cls_off[it->second + 1] : ft.pool.size()) - o;
            if (len == words.size() && std::memcmp(&ft.pool[o], words.data(), len * sizeof(int32_t)) == 0) cls = it->second;
        }
        if (cls < 0) {
            cls = (int32_t)ft.cls_off.size();
            ft.cls_off.push_back((int32_t)ft.pool.size());
            ft.pool.insert(ft.pool.end(), words.begin(), words.end());
            seen.emplace(hk, cls);
        }
        ft.tile_cls.push_back(cls);
    }
    return ft;
}

}  // namespace abl
