// Host-side check of the device layout's set-up (ablate_b200/csrc/fv_setup.hpp), compiled with g++ by
// tests/test_setup_records.py: reads a mesh descriptor from a binary file, builds the host mesh, the
// tiles and the cone-weight and face-geometry records with and without record tables, and checks
//   * the canonical cone order: each cell's neighbour offsets x_n - x_c ascend lexicographically;
//   * that the tables expand back to the one-record-per-item arrays bit for bit;
//   * that the fused kernel's per-tile tables (ext cells, local cones, faces and face lists, shared
//     between tiles whose tables are equal) decode back to the global mesh, tile by tile.
// Prints "weight_classes <n> geometry_classes <m> fused_classes <k> max_ext <e> ok <0|1>".
//
// File layout (little-endian): int32 dim, n_cells, n_faces, has_shift, lsq, dif; then face_cells
// (int32 [n_faces][2]), face_normal, face_centroid ([n_faces][3] double), cell_centroid ([n_cells][3]),
// cell_volume ([n_cells]), cell_kind (uint8 [n_cells]) and, when has_shift, face_shift ([n_faces][3]).
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fv_setup.hpp"

template <class T>
static bool read_array(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[6];
    if (std::fread(hdr, sizeof(int32_t), 6, f) != 6) return 2;
    const int dim = hdr[0], nc = hdr[1], nf = hdr[2];
    const bool has_shift = hdr[3] != 0, lsq = hdr[4] != 0, dif = hdr[5] != 0;
    std::vector<int32_t> fc;
    std::vector<double> fn, fcen, cc, cvol, fs;
    std::vector<uint8_t> ck;
    bool ok = read_array(f, fc, 2 * (size_t)nf) && read_array(f, fn, 3 * (size_t)nf) && read_array(f, fcen, 3 * (size_t)nf) &&
              read_array(f, cc, 3 * (size_t)nc) && read_array(f, cvol, (size_t)nc) && read_array(f, ck, (size_t)nc) &&
              (!has_shift || read_array(f, fs, 3 * (size_t)nf));
    std::fclose(f);
    if (!ok) return 2;
    abl_mesh_desc m{dim, nc, nf, fc.data(), fn.data(), fcen.data(), cc.data(), cvol.data(), ck.data(), has_shift ? fs.data() : nullptr};

    const abl::HostMesh h = abl::build_host_mesh(&m, lsq, dif);
    const abl::ConeRecords one = abl::cone_records(h, lsq, dif, false);
    const abl::ConeRecords tab = abl::cone_records(h, lsq, dif, true);
    bool pass = one.base.empty() && one.classes == 0;

    // canonical order: the offsets x_n - x_c of each cell (periodic images resolved) ascend
    auto offset = [&](int c, int i) {
        std::vector<double> v(3, 0.0);
        const size_t fi = (size_t)h.cone_face[i];
        for (int d = 0; d < dim; d++) {
            const double sh = has_shift ? fs[3 * fi + d] : 0.0;
            v[d] = cc[3 * (size_t)h.cone_nbr[i] + d] + (h.cone_side[i] == 0 ? sh : -sh) - cc[3 * (size_t)c + d];
        }
        return v;
    };
    for (int c = 0; c < nc && pass; c++)
        for (int i = h.cone_ptr[c] + 1; i < h.cone_ptr[c + 1] && pass; i++) pass = !(offset(c, i) < offset(c, i - 1));
    // the weight tables expand to the per-entry arrays bit for bit
    if (pass && tab.classes) {
        pass = tab.base.size() == (size_t)nc;
        for (int c = 0; c < nc && pass; c++)
            for (int k = 0; k < h.cone_ptr[c + 1] - h.cone_ptr[c] && pass; k++) {
                const size_t e = (size_t)(h.cone_ptr[c] + k), t = (size_t)tab.base[c] + k;
                pass = std::memcmp(&one.cwa[6 * e], &tab.cwa[6 * t], 6 * sizeof(double)) == 0 &&
                       std::memcmp(&one.cv[3 * e], &tab.cv[3 * t], 3 * sizeof(double)) == 0 &&
                       std::memcmp(&one.cwar[6 * e], &tab.cwar[6 * t], 6 * sizeof(double)) == 0;
            }
    } else if (pass) {
        pass = tab.cwa == one.cwa && tab.cv == one.cv && tab.cwar == one.cwar;
    }

    const abl::Tiles tl = abl::build_tiles(h, &m, 256, true);
    const abl::GeoRecords g1 = abl::tile_geometry(tl, false);
    const abl::GeoRecords gt = abl::tile_geometry(tl, true);
    const size_t ntf = tl.tf_cells.size() / 2;
    pass = pass && g1.cls.empty() && g1.geo.size() == 10 * ntf;
    if (pass && !gt.cls.empty()) {
        pass = gt.cls.size() == ntf;
        for (size_t i = 0; i < ntf && pass; i++)
            pass = (size_t)gt.cls[i] * 10 < gt.geo.size() &&
                   std::memcmp(&g1.geo[10 * i], &gt.geo[10 * (size_t)gt.cls[i]], 10 * sizeof(double)) == 0;
    } else if (pass) {
        pass = gt.geo == g1.geo;
    }

    // the fused tables, decoded tile by tile against the global mesh
    std::vector<int32_t> wb(nc);
    for (int c = 0; c < nc; c++) wb[c] = tab.classes ? tab.base[c] : h.cone_ptr[c];
    const abl::FusedTiles ft = abl::fused_tiles(h, tl, wb, gt.cls);
    pass = pass && (int)ft.tile_cls.size() == tl.n_tiles && (int)ft.ext_ptr.size() == tl.n_tiles + 1;
    for (int k = 0; k < tl.n_tiles && pass; k++) {
        const int32_t* cl = ft.pool.data() + ft.cls_off[ft.tile_cls[k]];
        const int nt = cl[0], ng = cl[1], ne = cl[2], nf = cl[3];
        const int32_t* gofs = cl + 4;
        const int32_t* wbs = gofs + ng + 1;
        const int32_t* kinds = wbs + ng;
        const int32_t* nbr = kinds + ng;
        const int32_t* faces = nbr + gofs[ng];
        const int32_t* fgeo = faces + nf;
        const int32_t* tcp = fgeo + nf;
        const int32_t* tce = tcp + nt + 1;
        const int32_t* ext = ft.ext.data() + ft.ext_ptr[k];
        const int cb = tl.cell_ptr[k], fb = tl.face_ptr[k];
        pass = nt == tl.cell_ptr[k + 1] - cb && nf == tl.face_ptr[k + 1] - fb && ne == ft.ext_ptr[k + 1] - ft.ext_ptr[k] && nt <= ng && ng <= ne;
        for (int j = 0; j < nt && pass; j++) pass = ext[j] == tl.cells[cb + j];
        for (int j = 0; j < ng && pass; j++) {
            const int c = ext[j];
            pass = gofs[j + 1] - gofs[j] == h.cone_ptr[c + 1] - h.cone_ptr[c] && wbs[j] == wb[c] && kinds[j] == h.kind[c];
            for (int i = 0; i < gofs[j + 1] - gofs[j] && pass; i++) {
                const int e = h.cone_ptr[c] + i, w = nbr[gofs[j] + i];
                pass = (w & 0xffff) < ne && ext[w & 0xffff] == h.cone_nbr[e] && ((w >> 16) != 0) == (h.face_boundary[h.cone_face[e]] != 0);
            }
        }
        // the faces are the tile's face records in another order: compare (left, right, geometry) multisets
        std::vector<std::array<int, 3>> a, b;
        for (int i = 0; i < nf && pass; i++) {
            const int lr = faces[i];
            pass = (lr & 0xffff) < ng && (lr >> 16) < ng;
            if (pass) a.push_back({ext[lr & 0xffff], ext[lr >> 16], fgeo[i]});
        }
        for (int i = 0; i < nf && pass; i++)
            b.push_back({tl.tf_cells[2 * (size_t)(fb + i)], tl.tf_cells[2 * (size_t)(fb + i) + 1], gt.cls.empty() ? fb + i : (int)gt.cls[fb + i]});
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        pass = pass && a == b;
        // each tile cell lists each of its faces once, on its own side, opposite faces next to each other
        for (int j = 0; j < nt && pass; j++) {
            const int c = ext[j];
            pass = tcp[j + 1] - tcp[j] == h.cone_ptr[c + 1] - h.cone_ptr[c];
            std::vector<int> seenf;
            for (int e = tcp[j]; e < tcp[j + 1] && pass; e++) {
                const int code = tce[e], fi = code & 0x7fff, lr = faces[fi];
                pass = fi < nf && ext[(code & 0x8000) ? (lr >> 16) : (lr & 0xffff)] == c &&
                       std::find(seenf.begin(), seenf.end(), fi) == seenf.end();
                seenf.push_back(fi);
            }
        }
    }
    std::printf("weight_classes %zu geometry_classes %zu fused_classes %zu max_ext %d ok %d\n", tab.classes,
                gt.cls.empty() ? (size_t)0 : gt.geo.size() / 10, ft.cls_off.size(), ft.max_ext, pass ? 1 : 0);
    return pass ? 0 : 1;
}
