// fv_fused.cuh -- the one-pass RHS (sm_100a): one CTA per tile of owned cells computes, from rows it
// stages in shared memory once,
//   1. the limited least-squares gradient and the aux gradient of every tile cell and of every cell
//      across a tile face ("ring 1"), whose stencils reach one ring further ("ring 2")
//      (CellInterpolant::ComputeFieldGradients + DMPlexApplyLimiter_Internal,
//      src/finiteVolume/cellInterpolant.cpp:282-497; the aux gradients FaceInterpolant averages,
//      src/finiteVolume/faceInterpolant.cpp:109-249);
//   2. the flux of every face of the tile (ComputeFluxSourceTerms, cellInterpolant.cpp:499-639, and the
//      process flux functions), with the same face_flux arithmetic as the two-pass kernels;
//   3. the residual of every tile cell: its signed face fluxes summed in ascending face order, scaled
//      by 1/V once and added into F (the reference's serial scatter made a per-cell gather).
// No gradient row goes to HBM: the state is read once per tile (ring cells again from L2), the residual
// written once. The ring gradients are computed by every tile that borders them; on an 8x8x4 tile of
// a hex box that doubles the gradient arithmetic, which costs less than writing and re-reading the
// gradient rows of the whole mesh.
//
// The per-tile tables (ext cells, local cones, local face cells, face lists) are built on the host by
// fused_tiles() (fv_setup.hpp); tiles whose tables are equal word for word share one copy, so a
// structured block reads its topology from a few kilobytes that stay in L1/L2.
#pragma once
#include "fv_kernels.cuh"

namespace abl {

constexpr int kFusedThreads = 512;

// device view of the fused tile tables
struct FusedDev {
    int max_ext, max_grad, max_faces;  // per-tile maxima (shared memory is sized by them)
    const int* ext_ptr;                // [n_tiles + 1] into ext
    const int* ext;                    // global cell of every ext slot: tile cells, ring 1, ring 2
    const int* tile_cls;               // [n_tiles] class of the tile's local tables
    const int* cls_off;                // [n_classes] offset of the class in pool
    const int* pool;                   // class tables (layout in fused_tiles())
};

// Shared-memory bytes of one CTA of the fused kernel: staged state rows (and the mixture's aux rows),
// gradient rows of gsize-byte elements padded to 16 bytes, one flux row per face.
__host__ __device__ inline size_t fused_smem_bytes(int dim, int nc, int naux, int gsize, int max_ext, int max_grad, int max_faces, bool nasa) {
    const int v = 16 / gsize;
    const int gw = (nc * dim + v - 1) / v * v + (naux * dim + v - 1) / v * v;
    size_t w = (size_t)max_ext * nc + (nasa ? (size_t)max_ext * naux : 0);  // doubles
    w = (w + 1) & ~size_t(1);                                                 // 16-byte rows below
    size_t bytes = w * sizeof(double) + (size_t)max_grad * gw * gsize;
    bytes = (bytes + 15) & ~size_t(15);
    return bytes + (size_t)max_faces * nc * sizeof(double);
}
constexpr size_t kFusedSmemLimit = 227 * 1024;

// The rows of the face flux from shared memory, by tile-local slot (the counterpart of GlobalRows).
template <int DIM, int NS, class G>
struct SharedRows {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, G>;
    static constexpr int GW = GR::GS + GR::AS;
    const double* sU;  // [slot][NC]
    const double* sA;  // [slot][NA] (mixture EOS)
    const G* sG;       // [slot][GW]: limited state gradient, then aux gradient
    bool nasa;
    template <class S>
    __device__ __forceinline__ void state(int c, S* u) const {
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) u[k] = sU[(size_t)c * D::NC + k];
    }
    __device__ __forceinline__ double temperature(int c) const { return sA[(size_t)c * D::NA]; }
    template <class S>
    __device__ __forceinline__ void aux_of(const Phys& P, const S* u, int c, S* a) const {
        if (NS > 0 && nasa) {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) a[k] = sA[(size_t)c * D::NA + k];
        } else {
            aux_from_state<DIM, NS>(P, u, a);
        }
    }
    template <int N>
    __device__ __forceinline__ void row(const G* p, G* out) const {
        if constexpr (sizeof(G) == 8) {
ABL_UNROLL_SPECIES
            for (int i = 0; i < N / 2; i++) {
                const double2 v = reinterpret_cast<const double2*>(p)[i];
                out[2 * i] = v.x;
                out[2 * i + 1] = v.y;
            }
            if constexpr (N % 2) out[N - 1] = p[N - 1];
        } else {
ABL_UNROLL_SPECIES
            for (int i = 0; i < N / 4; i++) {
                const float4 v = reinterpret_cast<const float4*>(p)[i];
                out[4 * i] = v.x;
                out[4 * i + 1] = v.y;
                out[4 * i + 2] = v.z;
                out[4 * i + 3] = v.w;
            }
ABL_UNROLL_SPECIES
            for (int i = (N / 4) * 4; i < N; i++) out[i] = p[i];
        }
    }
    __device__ __forceinline__ void grad_row(int c, G* g) const { row<D::NC * DIM>(sG + (size_t)c * GW, g); }
    __device__ __forceinline__ void agrad_row(int c, G* g) const { row<D::NA * DIM>(sG + (size_t)c * GW + GR::GS, g); }
};

// Limiter of one field (components k0..k1-1) of a gradient cell, neighbour states from shared memory:
// the arithmetic of limit_field() in its non-recording form, in the same order.
template <int DIM, int NS, class G, int LIM>
__device__ __forceinline__ void limit_field_shared(const DevMesh& M, const Phys& P, const double* sU, const int* nbr, int beg, int end,
                                                   size_t wb, const double* uc, G* g, int k0, int k1) {
    using D = Dims<DIM, NS>;
    G phi[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) phi[k] = big_value<G>();
#pragma unroll 1
    for (int i = beg; i < end; i++) {
        G v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) v[d] = geo<G>(M.cv, M.cv32, 3 * (wb + (size_t)(i - beg)) + d);
        const double* un = sU + (size_t)(__ldg(nbr + i) & 0xffff) * D::NC;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            if (k < k0 || k >= k1) continue;
            G denom = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) denom += g[k * DIM + d] * v[d];
            const G diff = G(un[k] - uc[k]);
            const G flim = G(0.5) * diff * rcp64(denom);
            phi[k] = pmin(phi[k], limiter_k<LIM, G>(P.limiter, flim));
        }
    }
    bool cancel = false;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
        if (phi[k] == G(0)) {
#pragma unroll
            for (int d = 0; d < DIM; d++)
                if (dabs(g[k * DIM + d]) > G(P.max_lim_grad)) cancel = true;
        }
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
#pragma unroll
        for (int d = 0; d < DIM; d++) g[k * DIM + d] *= cancel ? G(0) : phi[k];
    }
}

// Gradient row of ext slot j (a tile or ring-1 cell): the arithmetic of k_gradient, in the same order,
// from the staged rows. kind, the cone entries [beg, end) of the class's neighbour list (local slot |
// boundary-face flag << 16) and the weight record base wb come from the class tables.
template <int DIM, int NS, class G, int LIM>
__device__ __forceinline__ void fused_gradient(const DevMesh& M, const Phys& P, const SharedRows<DIM, NS, G>& src, G* out, int j, int kind,
                                               const int* nbr, int beg, int end, size_t wb, int do_state, int do_aux) {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, G>;
    const bool state = do_state && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO);
    const bool auxg = do_aux && kind != ABL_CELL_HALO_OUTER;
    double uc[D::NC], ac[D::NA];
    src.state(j, uc);
    if (auxg) src.aux_of(P, uc, j, ac);
    G g[D::NC * DIM], ga[D::NA * DIM];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC * DIM; k++) g[k] = G(0);
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA * DIM; k++) ga[k] = G(0);
    if (state || auxg) {
#pragma unroll 1
        for (int i = beg; i < end; i++) {
            const int nb = __ldg(nbr + i);
            const int n = nb & 0xffff;
            double un[D::NC];
            src.state(n, un);
            G wd[DIM], wad[DIM];
            cone_weights<DIM, G>(M.cwa, M.cwa32, wb + (size_t)(i - beg), wd, wad);
            if (state && !(nb >> 16)) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) {
                    const G delta = G(un[k] - uc[k]);
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[k * DIM + d] += wd[d] * delta;
                }
            }
            if (auxg) {
                double an[D::NA];
                src.aux_of(P, un, n, an);
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NA; k++) {
                    const G delta = G(an[k] - ac[k]);
#pragma unroll
                    for (int d = 0; d < DIM; d++) ga[k * DIM + d] += wad[d] * delta;
                }
            }
        }
        if (state && P.limiter != ABL_LIMITER_NONE) {
            limit_field_shared<DIM, NS, G, LIM>(M, P, src.sU, nbr, beg, end, wb, uc, g, 0, D::NE);
            if (NS > 0) limit_field_shared<DIM, NS, G, LIM>(M, P, src.sU, nbr, beg, end, wb, uc, g, D::NE, D::NC);
        }
    }
    if (do_state) {
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC * DIM; k++) out[k] = g[k];
    }
    if (do_aux) {
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NA * DIM; k++) out[GR::GS + k] = ga[k];
    }
}

// One CTA per tile, persistent over the tiles [t0, t1) (CTA b takes tiles t0 + b, t0 + b + gridDim.x, ...).
// Class table layout (int words, from the class's offset in the pool):
//   n_t, n_g, n_e, n_f                         tile cells, gradient cells (tile + ring 1), ext slots, faces
//   gofs[n_g + 1]                              start of each gradient cell's cone in nbr
//   wb[n_g]                                    first weight record of each gradient cell's cone
//   kind[n_g]                                  cell kind
//   nbr[gofs[n_g]]                             neighbour slot | boundary-face flag << 16
//   face[n_f]                                  left slot | right slot << 16
//   fgeo[n_f]                                  geometry record of the face
//   tcp[n_t + 1], tce[tcp[n_t]]                per tile cell its faces: local face | side << 15
template <int DIM, int NS, class G, int FK, int LIM>
__global__ void __launch_bounds__(kFusedThreads, 1)
    k_fused_rhs(DevMesh M, Phys P, FusedDev T, const double* __restrict__ U, const double* __restrict__ aux, double* __restrict__ F,
                int overwrite, int do_state, int do_aux, int* status, int t0, int t1) {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, G>;
    constexpr int GW = GR::GS + GR::AS;
    extern __shared__ __align__(16) unsigned char fsm[];
    const bool nasa = NS > 0 && P.eos == ABL_EOS_NASA7;
    double* sU = reinterpret_cast<double*>(fsm);
    double* sA = sU + (size_t)T.max_ext * D::NC;
    size_t w = (size_t)T.max_ext * D::NC + (nasa ? (size_t)T.max_ext * D::NA : 0);
    w = (w + 1) & ~size_t(1);
    G* sG = reinterpret_cast<G*>(sU + w);
    double* sF = reinterpret_cast<double*>(fsm + ((w * sizeof(double) + (size_t)T.max_grad * GW * sizeof(G) + 15) & ~size_t(15)));
    const SharedRows<DIM, NS, G> src{sU, sA, sG, nasa};
    bool ok = true, rok = true, finite = true;
    for (int t = t0 + blockIdx.x; t < t1; t += gridDim.x) {
        const int* cl = T.pool + __ldg(T.cls_off + __ldg(T.tile_cls + t));
        const int nt = __ldg(cl), ng = __ldg(cl + 1), ne = __ldg(cl + 2), nf = __ldg(cl + 3);
        const int* gofs = cl + 4;
        const int* wbs = gofs + ng + 1;
        const int* kinds = wbs + ng;
        const int* nbr = kinds + ng;
        const int* faces = nbr + __ldg(gofs + ng);
        const int* fgeo = faces + nf;
        const int* tcp = fgeo + nf;
        const int* tce = tcp + nt + 1;
        const int* ext = T.ext + __ldg(T.ext_ptr + t);
        // stage: the state row (and the mixture's aux row) of every ext slot, consecutive threads on
        // consecutive doubles of a row
        for (int e = threadIdx.x; e < ne * D::NC; e += blockDim.x) {
            const int s = e / D::NC;
            sU[e] = __ldg(U + (size_t)__ldg(ext + s) * D::NC + (e - s * D::NC));
        }
        if (nasa) {
            for (int e = threadIdx.x; e < ne * D::NA; e += blockDim.x) {
                const int s = e / D::NA;
                sA[e] = __ldg(aux + (size_t)__ldg(ext + s) * D::NA + (e - s * D::NA));
            }
        }
        __syncthreads();
        if (do_state || do_aux) {
            for (int j = threadIdx.x; j < ng; j += blockDim.x)
                fused_gradient<DIM, NS, G, LIM>(M, P, src, sG + (size_t)j * GW, j, __ldg(kinds + j), nbr, __ldg(gofs + j), __ldg(gofs + j + 1),
                                                (size_t)__ldg(wbs + j), do_state, do_aux);
            __syncthreads();
        }
        for (int i = threadIdx.x; i < nf; i += blockDim.x) {
            const int lr = __ldg(faces + i);
            double normal[DIM], fdx[6];
            face_geometry_rec<DIM, G>(M, (size_t)__ldg(fgeo + i), normal, fdx);
            double flux[D::NC];
            face_flux<DIM, NS, G, FK>(P, src, lr & 0xffff, (int)((unsigned)lr >> 16), normal, fdx, flux, &ok, &rok);
            double* out = sF + (size_t)i * D::NC;
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) out[k] = flux[k];
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            const int c = __ldg(ext + j);
            const double iv = __ldg(M.ivol + c);
            // the signed face fluxes summed first, then scaled by 1/V once (as k_tile_flux)
            double sum[D::NC];
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) sum[k] = 0.0;
            const int e0 = __ldg(tcp + j), e1 = __ldg(tcp + j + 1);
            for (int e = e0; e < e1; e++) {
                const int code = __ldg(tce + e);
                const double* ff = sF + (size_t)(code & 0x7fff) * D::NC;
                if (code & 0x8000) {
ABL_UNROLL_SPECIES
                    for (int k = 0; k < D::NC; k++) sum[k] += ff[k];
                } else {
ABL_UNROLL_SPECIES
                    for (int k = 0; k < D::NC; k++) sum[k] -= ff[k];
                }
            }
            double* Fc = F + (size_t)c * D::NC;
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) {
                const double acc = (overwrite ? 0.0 : Fc[k]) + sum[k] * iv;
                Fc[k] = acc;
                finite = finite && dfinite(acc);
            }
        }
        __syncthreads();  // the next tile overwrites the staged rows
    }
    if (!finite) atomicOr(status, kStatusNaN);
    if (!ok) atomicOr(status, kStatusEos);
    if (!rok) atomicOr(status, kStatusRiemann);
}

}  // namespace abl
