// fv_handle.hpp -- host-side state of one abl_fv handle and the helpers the ABI and launch code share.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "fv_adjoint.cuh"
#include "fv_fused.cuh"

namespace abl {

extern thread_local std::string g_last_error;

struct AblError : std::runtime_error {
    int code;
    AblError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define ABL_CUDA(call)                                                                                           \
    do {                                                                                                         \
        cudaError_t e_ = (call);                                                                                 \
        if (e_ != cudaSuccess) throw AblError(ABL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw AblError(e == cudaErrorMemoryAllocation ? ABL_ERR_OUT_OF_MEMORY : ABL_ERR_CUDA,
                           std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
    }
    void upload(const T* h, size_t count) {
        alloc(count);
        if (count) ABL_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    void zero() {
        if (n) ABL_CUDA(cudaMemset(p, 0, n * sizeof(T)));
    }
};

inline unsigned blocks_for(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

inline void check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw AblError(ABL_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

// gradient rows are padded to whole 16-byte vectors (see GradRows in fv_kernels.cuh)
inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace abl

struct abl_fv {
    int device = 0;
    int dim = 0, ns = 0, nc = 0, naux = 0;  // of the compiled instance that runs (species capacity)
    // the caller's species count and row widths; pad = ns - ns_user zero-state species sit in front of
    // the caller's species in the instance's rows (0: the count has an instance of its own)
    int ns_user = 0, nc_user = 0, naux_user = 0, pad = 0;
    abl::DevBuf<double> pU, pdU, pF, pdF, pUb;  // rows in the instance's width when pad > 0
    int n_cells = 0, n_faces = 0, n_flux_faces = 0;
    abl::Phys phys{};
    abl::DevMesh mesh{};
    // resident mesh + geometry
    abl::DevBuf<int2> face_cells, cone;
    abl::DevBuf<uint8_t> kind;
    abl::DevBuf<int> cone_ptr;
    abl::DevBuf<double> fdx, ivol, cgrad, fgrad;
    abl::DevBuf<double> nasa7, mw, inv_mw, href, diff_k;
    // tiles
    abl::DevBuf<int> tile_cell_ptr, tile_cells, tile_face_ptr, tc_fptr;
    abl::DevBuf<int2> tf_cells;
    abl::DevBuf<double> tf_geo, tf_geo32;
    abl::DevBuf<uint16_t> tf_gcls;  // per tile face record, its geometry record (when they repeat)
    int n_geo_classes = 0;          // 0: one geometry record per tile face record
    abl::DevBuf<uint16_t> tc_face;
    int tile_smem = 0;
    // adjoint: tile face colours and slots, non-owned records
    abl::DevBuf<int> col_base, col_start, tf_nb, face_nb, nonowned;
    abl::DevBuf<uint32_t> tf_slot;
    abl::DevBuf<uint16_t> tf_adj;
    int tile_max_cells = 0, n_nb = 0;
    // the fused one-pass RHS: per-tile ext cells and class tables; usable per gradient precision
    // (0: FP64, 1: mixed) when a tile's rows fit in shared memory
    abl::DevBuf<int> fz_ext_ptr, fz_ext, fz_tile_cls, fz_cls_off, fz_pool;
    int fz_max_ext = 0, fz_max_grad = 0, fz_max_faces = 0, fz_classes = 0;
    bool fused_ok[2] = {false, false};
    // a mixed request with species runs the FP32-gradient kernels (ABL_FV_MIXED_SPECIES=1 at create)
    bool mixed_species = false;
    size_t fused_smem[2] = {0, 0};
    int n_sm = 1;
    // optional per-kernel timing of the last evaluation
    bool profile = false;
    int n_marks = 0;
    cudaEvent_t marks[8] = {};
    const char* mark_names[8] = {};
    // work buffers: aux, gradients (FP64, FP32, and value+tangent pairs for the tangent kernels)
    abl::DevBuf<double> aux;
    abl::DevBuf<double> grad64, agrad64, gradD, agradD;
    abl::DevBuf<float> grad32, agrad32;
    abl::DevBuf<int> status;
    // adjoint work buffers, allocated on the first VJP
    abl::DevBuf<double> adj_gb, adj_beta, adj_gab, adj_ub, adj_ab, adj_nb, adj_graw, adj_phi;
    abl::DevBuf<int> adj_fstar, adj_ist;
    abl::DevBuf<double> wsum, cwa, cv, cwar;
    abl::DevBuf<float> cwa32, cv32;
    abl::DevBuf<int> cone_cls;  // per cell, the first entry of its weight sequence (when they repeat)
    int n_cone_classes = 0;     // 0: one weight record per cone entry
    int max_cone = 0;
    // boundary ghosts and time stepping
    int n_ghost = 0;
    abl::DevBuf<int> ghost_cell, ghost_nbr, ghost_bc;
    abl::DevBuf<double> ghost_normal, rmin;
    abl::DevBuf<abl_bc> bc_table;
    abl::DevBuf<unsigned long long> dt_bits;
    abl::DevBuf<double> step_U1, step_F;
    // ghosts grouped by interior neighbour (adjoint of the fill), per-ghost value adjoints
    int n_gseg = 0;
    abl::DevBuf<int> gseg_ptr, gseg_nbr, gseg_ghost;
    // owned rows in ascending local order (the rank's part of the PETSc global vector) and a staging buffer
    abl::DevBuf<int> owned_rows;
    abl::DevBuf<double> io_rows;
    abl::DevBuf<double> ghost_vbar, bc_vbar;
    int n_bc = 1;
    // wall-pressure functional: distinct cells, weights, per-block partial sums
    int fn_n = 0;
    abl::DevBuf<int> fn_cells;
    abl::DevBuf<double> fn_w, fn_partial;
    // host-pointer paths
    abl::DevBuf<double> hU, hF, hdU, hdF;
    // host-buffer RHS pipeline: after the state, F comes in on a copy stream while the gradient pass
    // runs, chunk by chunk, each tile chunk waiting for its own rows; finished chunks go out on a third
    // stream (the other copy direction) while the next ones run (when the tiles' cells are row ranges)
    static constexpr int kHostChunks = 16;
    cudaStream_t host_stream = nullptr, copy_stream = nullptr, out_stream = nullptr;
    cudaEvent_t ev_u = nullptr, ev_in[kHostChunks] = {}, ev_chunk[kHostChunks] = {};
    int owned_lo = 0, owned_hi = -1;   // owned rows are [owned_lo, owned_hi) when contiguous, else owned_hi = -1
    std::vector<int> chunk_tile;       // tile boundaries of the output chunks (empty: one copy after the pass)
    std::vector<int> chunk_row;        // their row boundaries
    bool pipe_active = false;          // set for the duration of one abl_fv_rhs_host call
    double* pipe_F_host = nullptr;
    bool need_aux = false, need_state_grad = false, need_aux_grad = false;
    // split RHS (abl_fv_rhs_phase): -1 the whole RHS; 0 the aux update and gradients of the cells whose
    // stencils hold no halo row; 1 the rest. Cell lists of the two parts:
    int rhs_phase = -1;
    abl::DevBuf<int> aux_early, aux_late, grad_early, grad_late;
};

namespace abl {

// record a timing mark (event) before the next launch when profiling is on
inline void mark(abl_fv* fv, const char* name, cudaStream_t s) {
    if (!fv->profile || fv->n_marks >= 8) return;
    if (!fv->marks[fv->n_marks]) ABL_CUDA(cudaEventCreate(&fv->marks[fv->n_marks]));
    ABL_CUDA(cudaEventRecord(fv->marks[fv->n_marks], s));
    fv->mark_names[fv->n_marks] = name;
    fv->n_marks++;
}

// launch sequences, explicitly instantiated per (DIM, NS) in fv_inst_*.cu
template <int DIM, int NS>
void run_rhs(abl_fv* fv, const double* U, double* F, int precision, int overwrite, cudaStream_t s);
template <int DIM, int NS>
void run_aux(abl_fv* fv, const double* U, cudaStream_t s);
template <int DIM, int NS>
void run_jvp(abl_fv* fv, const double* U, const double* dU, double* F, double* dF, cudaStream_t s);
template <int DIM, int NS>
void run_vjp(abl_fv* fv, const double* U, const double* Fb, double* Ub, cudaStream_t s);

}  // namespace abl
