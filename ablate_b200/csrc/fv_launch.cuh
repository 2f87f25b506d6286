// fv_launch.cuh -- the launch sequences of one RHS / aux update / tangent evaluation for a compiled
// (DIM, NS) instance. Included only by the fv_inst_*.cu translation units, which instantiate them.
#pragma once
#include "fv_handle.hpp"

namespace abl {

template <int DIM, int NS, class G, int FK>
void launch_tile(abl_fv* fv, const double* U, const double* dU, const G* grad, const G* agrad, double* F, double* dF, int overwrite,
                 cudaStream_t s) {
    auto kern = k_tile_flux<DIM, NS, G, FK>;
    const int smem = fv->tile_smem * (std::is_same<G, Dual>::value ? 2 : 1);
    if (smem > 227 * 1024) throw AblError(ABL_ERR_UNSUPPORTED, "tile flux buffer exceeds shared memory for this species count");
    ABL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (!fv->pipe_active) {
        kern<<<fv->mesh.n_tiles, 128, smem, s>>>(fv->mesh, fv->phys, U, dU, fv->aux.p, grad, agrad, F, dF, overwrite, fv->status.p, 0);
        check_launch();
        return;
    }
    // host-buffer call: each chunk of tiles waits for its residual rows, and once done sends them back on
    // the output stream while the next chunk runs
    const int nch = fv->chunk_tile.empty() ? 0 : (int)fv->chunk_tile.size() - 1;
    if (nch == 0) {
        ABL_CUDA(cudaStreamWaitEvent(s, fv->ev_in[0], 0));
        kern<<<fv->mesh.n_tiles, 128, smem, s>>>(fv->mesh, fv->phys, U, dU, fv->aux.p, grad, agrad, F, dF, overwrite, fv->status.p, 0);
        check_launch();
        return;
    }
    for (int q = 0; q < nch; q++) {
        const int ta = fv->chunk_tile[q], tb = fv->chunk_tile[q + 1];
        ABL_CUDA(cudaStreamWaitEvent(s, fv->ev_in[q], 0));
        if (tb > ta) {
            kern<<<tb - ta, 128, smem, s>>>(fv->mesh, fv->phys, U, dU, fv->aux.p, grad, agrad, F, dF, overwrite, fv->status.p, ta);
            check_launch();
        }
        ABL_CUDA(cudaEventRecord(fv->ev_chunk[q], s));
        ABL_CUDA(cudaStreamWaitEvent(fv->out_stream, fv->ev_chunk[q], 0));
        const size_t r0 = (size_t)fv->chunk_row[q] * fv->nc, r1 = (size_t)fv->chunk_row[q + 1] * fv->nc;
        if (r1 > r0)
            ABL_CUDA(cudaMemcpyAsync(fv->pipe_F_host + r0, F + r0, (r1 - r0) * sizeof(double), cudaMemcpyDeviceToHost, fv->out_stream));
    }
}

// the fused one-pass RHS over all tiles, or (host-buffer call) chunk by chunk as launch_tile does
template <int DIM, int NS, class G, int FK, int LIM>
void launch_fused(abl_fv* fv, const double* U, double* F, int overwrite, cudaStream_t s) {
    auto kern = k_fused_rhs<DIM, NS, G, FK, LIM>;
    const int q = std::is_same<G, float>::value ? 1 : 0;
    const size_t smem = fv->fused_smem[q];
    ABL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const FusedDev T{fv->fz_max_ext, fv->fz_max_grad, fv->fz_max_faces, fv->fz_ext_ptr.p, fv->fz_ext.p, fv->fz_tile_cls.p, fv->fz_cls_off.p,
                     fv->fz_pool.p};
    auto run = [&](int ta, int tb) {
        if (tb <= ta) return;
        // persistent: one CTA per SM (the shared memory of a tile allows one), each looping over tiles
        const int grid = std::min(tb - ta, fv->n_sm);
        kern<<<grid, kFusedThreads, smem, s>>>(fv->mesh, fv->phys, T, U, fv->aux.p, F, overwrite, fv->need_state_grad, fv->need_aux_grad,
                                               fv->status.p, ta, tb);
        check_launch();
    };
    if (!fv->pipe_active) {
        run(0, fv->mesh.n_tiles);
        return;
    }
    const int nch = fv->chunk_tile.empty() ? 0 : (int)fv->chunk_tile.size() - 1;
    if (nch == 0) {
        ABL_CUDA(cudaStreamWaitEvent(s, fv->ev_in[0], 0));
        run(0, fv->mesh.n_tiles);
        return;
    }
    for (int c = 0; c < nch; c++) {
        const int ta = fv->chunk_tile[c], tb = fv->chunk_tile[c + 1];
        ABL_CUDA(cudaStreamWaitEvent(s, fv->ev_in[c], 0));
        run(ta, tb);
        ABL_CUDA(cudaEventRecord(fv->ev_chunk[c], s));
        ABL_CUDA(cudaStreamWaitEvent(fv->out_stream, fv->ev_chunk[c], 0));
        const size_t r0 = (size_t)fv->chunk_row[c] * fv->nc, r1 = (size_t)fv->chunk_row[c + 1] * fv->nc;
        if (r1 > r0)
            ABL_CUDA(cudaMemcpyAsync(fv->pipe_F_host + r0, F + r0, (r1 - r0) * sizeof(double), cudaMemcpyDeviceToHost, fv->out_stream));
    }
}

// shared memory for the neighbour differences the limiter reuses (none when it would not fit)
template <int DIM, int NS, class G>
size_t gradient_smem(const abl_fv* fv) {
    const size_t b = (size_t)128 * fv->mesh.max_cone * Dims<DIM, NS>::NC * sizeof(G);
    return b <= 48 * 1024 ? b : 0;
}

// the gradient pass over every cell, or (split RHS) over the phase's cells
template <int DIM, int NS, class G, int LIM>
void launch_gradient(abl_fv* fv, const double* U, const double* dU, G* grad, G* agrad, cudaStream_t s) {
    const size_t smem = gradient_smem<DIM, NS, G>(fv);
    const abl::DevBuf<int>* list = fv->rhs_phase == 0 ? &fv->grad_early : fv->rhs_phase == 1 ? &fv->grad_late : nullptr;
    const int n = list ? (int)list->n : fv->mesh.n_cells;
    if (n == 0) return;
    k_gradient<DIM, NS, G, LIM><<<blocks_for(n, 128), 128, smem, s>>>(fv->mesh, fv->phys, U, dU, fv->aux.p, grad, agrad, fv->need_state_grad,
                                                                   fv->need_aux_grad, smem > 0, nullptr, nullptr, nullptr, list ? list->p : nullptr, n);
    check_launch();
}

// the aux update over every cell, or (split RHS) over the phase's cells
template <int DIM, int NS>
void launch_aux(abl_fv* fv, const double* U, cudaStream_t s) {
    const abl::DevBuf<int>* list = fv->rhs_phase == 0 ? &fv->aux_early : fv->rhs_phase == 1 ? &fv->aux_late : nullptr;
    const int n = list ? (int)list->n : fv->mesh.n_cells;
    if (n == 0) return;
    k_aux<DIM, NS><<<blocks_for(n, 256), 256, 0, s>>>(fv->mesh, fv->phys, U, fv->aux.p, fv->status.p, list ? list->p : nullptr, n);
    check_launch();
}

// the RHS for gradient storage type G: limiter and flux calculator fixed at compile time where a
// specialised kernel exists (minmod; AUSM, AUSM+up), chosen at run time otherwise
template <int DIM, int NS, class G>
void rhs_with(abl_fv* fv, const double* U, G* grad, G* agrad, double* F, int overwrite, cudaStream_t s) {
    const Phys& P = fv->phys;
    if constexpr (!kSpecialized<NS>) {
        // a capacity instance: generic limiter and flux calculator
        if (fv->need_state_grad || fv->need_aux_grad) {
            mark(fv, "k_gradient", s);
            launch_gradient<DIM, NS, G, -1>(fv, U, nullptr, grad, agrad, s);
        }
        mark(fv, "k_tile_flux", s);
        if (fv->mesh.n_tiles > 0 && fv->rhs_phase != 0) launch_tile<DIM, NS, G, -1>(fv, U, nullptr, grad, agrad, F, nullptr, overwrite, s);
        return;
    } else if (fv->fused_ok[std::is_same<G, float>::value ? 1 : 0]) {
        // one pass over everything: nothing in the first phase of a split RHS
        if (fv->rhs_phase == 0) return;
        mark(fv, "k_fused_rhs", s);
        if (fv->mesh.n_tiles > 0) {
            if (P.flux == ABL_FLUX_AUSMPUP) {
                if (P.limiter == ABL_LIMITER_MINMOD)
                    launch_fused<DIM, NS, G, ABL_FLUX_AUSMPUP, ABL_LIMITER_MINMOD>(fv, U, F, overwrite, s);
                else
                    launch_fused<DIM, NS, G, ABL_FLUX_AUSMPUP, -1>(fv, U, F, overwrite, s);
            } else if (P.flux == ABL_FLUX_AUSM) {
                launch_fused<DIM, NS, G, ABL_FLUX_AUSM, -1>(fv, U, F, overwrite, s);
            } else {
                launch_fused<DIM, NS, G, -1, -1>(fv, U, F, overwrite, s);
            }
        }
        return;
    }
    if (fv->need_state_grad || fv->need_aux_grad) {
        mark(fv, "k_gradient", s);
        if (P.limiter == ABL_LIMITER_MINMOD)
            launch_gradient<DIM, NS, G, ABL_LIMITER_MINMOD>(fv, U, nullptr, grad, agrad, s);
        else
            launch_gradient<DIM, NS, G, -1>(fv, U, nullptr, grad, agrad, s);
    }
    mark(fv, "k_tile_flux", s);
    if (fv->mesh.n_tiles > 0 && fv->rhs_phase != 0) {
        if (P.flux == ABL_FLUX_AUSMPUP)
            launch_tile<DIM, NS, G, ABL_FLUX_AUSMPUP>(fv, U, nullptr, grad, agrad, F, nullptr, overwrite, s);
        else if (P.flux == ABL_FLUX_AUSM)
            launch_tile<DIM, NS, G, ABL_FLUX_AUSM>(fv, U, nullptr, grad, agrad, F, nullptr, overwrite, s);
        else
            launch_tile<DIM, NS, G, -1>(fv, U, nullptr, grad, agrad, F, nullptr, overwrite, s);
    }
}

template <int DIM, int NS>
void run_rhs(abl_fv* fv, const double* U, double* F, int precision, int overwrite, cudaStream_t s) {
    fv->n_marks = 0;
    if (fv->need_aux) {
        mark(fv, "k_aux", s);
        launch_aux<DIM, NS>(fv, U, s);
    }
    // With species a mixed request runs the FP64 kernels unless the handle was created with
    // ABL_FV_MIXED_SPECIES=1: the NASA-7 decode (FP64 by design) dominates their cost (the FP32-gradient
    // kernels gain 2-6 %), and on the 2M-tetrahedron channel their error reaches 1.2e-6 against FP64.
    bool done = false;
    if constexpr (kSpecialized<NS>) {
        if (precision == ABL_PRECISION_MIXED && (NS == 0 || fv->mixed_species)) {
            rhs_with<DIM, NS, float>(fv, U, fv->grad32.p, fv->agrad32.p, F, overwrite, s);
            done = true;
        }
    }
    if (!done) rhs_with<DIM, NS, double>(fv, U, fv->grad64.p, fv->agrad64.p, F, overwrite, s);
    mark(fv, "end", s);
}

template <int DIM, int NS>
void run_aux(abl_fv* fv, const double* U, cudaStream_t s) {
    k_aux<DIM, NS><<<blocks_for(fv->mesh.n_cells, 256), 256, 0, s>>>(fv->mesh, fv->phys, U, fv->aux.p, fv->status.p);
    check_launch();
}

// forward tangent: the FP64 RHS kernels evaluated on Dual numbers (value + one directional derivative)
template <int DIM, int NS>
void run_jvp(abl_fv* fv, const double* U, const double* dU, double* F, double* dF, cudaStream_t s) {
    const DevMesh& M = fv->mesh;
    fv->n_marks = 0;
    if (fv->need_aux) {
        mark(fv, "k_aux", s);
        k_aux<DIM, NS><<<blocks_for(M.n_cells, 256), 256, 0, s>>>(M, fv->phys, U, fv->aux.p, fv->status.p);
        check_launch();
    }
    Dual* grad = reinterpret_cast<Dual*>(fv->gradD.p);
    Dual* agrad = reinterpret_cast<Dual*>(fv->agradD.p);
    if (fv->need_state_grad || fv->need_aux_grad) {
        mark(fv, "k_gradient_tangent", s);
        launch_gradient<DIM, NS, Dual, -1>(fv, U, dU, grad, agrad, s);
    }
    mark(fv, "k_tile_flux_tangent", s);
    if (M.n_tiles > 0) launch_tile<DIM, NS, Dual, -1>(fv, U, dU, grad, agrad, F, dF, 0, s);
    mark(fv, "end", s);
}

// reverse mode: Ub += (dF/dU)^T Fb with the forward gradients recomputed (k_gradient), the face
// fluxes run backwards per tile, then the per-cell limiter / gradient / aux steps and their gather
template <int DIM, int NS>
void run_vjp(abl_fv* fv, const double* U, const double* Fb, double* Ub, cudaStream_t s) {
    using AR = AdjRow<DIM, NS>;
    const DevMesh& M = fv->mesh;
    const Phys& P = fv->phys;
    fv->n_marks = 0;
    if (fv->need_aux) {
        mark(fv, "k_aux", s);
        k_aux<DIM, NS><<<blocks_for(M.n_cells, 256), 256, 0, s>>>(M, P, U, fv->aux.p, fv->status.p);
        check_launch();
    }
    GradRec rec{fv->adj_graw.p, fv->adj_phi.p, fv->adj_ist.p};
    if (fv->need_state_grad || fv->need_aux_grad) {
        mark(fv, "k_gradient", s);
        auto kern = k_gradient<DIM, NS, double, -1, true>;
        if constexpr (kSpecialized<NS>)
            if (P.limiter == ABL_LIMITER_MINMOD) kern = k_gradient<DIM, NS, double, ABL_LIMITER_MINMOD, true>;
        const size_t smem = gradient_smem<DIM, NS, double>(fv);
        kern<<<blocks_for(M.n_cells, 128), 128, smem, s>>>(M, P, U, nullptr, fv->aux.p, fv->grad64.p, fv->agrad64.p, fv->need_state_grad,
                                                          fv->need_aux_grad, smem > 0, fv->adj_graw.p, fv->adj_phi.p, fv->adj_ist.p, nullptr, 0);
        check_launch();
    }
    AdjOut<DIM, NS> out{fv->need_state_grad ? fv->adj_gb.p : nullptr, fv->adj_beta.p, fv->adj_fstar.p,
                        fv->need_aux_grad ? fv->adj_gab.p : nullptr, fv->adj_ub.p, fv->adj_ab.p};
    const int ds = fv->need_state_grad, da = fv->need_aux_grad;
    mark(fv, "k_tile_adjoint", s);
    if (fv->n_nb > 0) ABL_CUDA(cudaMemsetAsync(fv->adj_nb.p, 0, (size_t)fv->n_nb * AR::N * sizeof(double), s));
    if (M.n_tiles > 0) {
        const size_t smem = (size_t)fv->tile_max_cells * AR::S * sizeof(double);
        if (smem > 227 * 1024) throw AblError(ABL_ERR_UNSUPPORTED, "adjoint accumulators exceed shared memory for this species count");
        // flux calculator and limiter fixed at compile time where a specialised kernel exists
        auto kern = k_tile_adjoint<DIM, NS, -1, -1>;
        if constexpr (kSpecialized<NS>) {
            if (P.flux == ABL_FLUX_AUSMPUP)
                kern = P.limiter == ABL_LIMITER_MINMOD ? k_tile_adjoint<DIM, NS, ABL_FLUX_AUSMPUP, ABL_LIMITER_MINMOD>
                                                       : k_tile_adjoint<DIM, NS, ABL_FLUX_AUSMPUP, -1>;
            else if (P.flux == ABL_FLUX_AUSM)
                kern = k_tile_adjoint<DIM, NS, ABL_FLUX_AUSM, -1>;
        }
        ABL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        static_assert(2 * kColorCap == 256, "one colour per pass of the 256-thread adjoint CTA");
        kern<<<M.n_tiles, 256, smem, s>>>(M, P, U, fv->aux.p, fv->grad64.p, fv->agrad64.p, Fb, rec, out, fv->adj_nb.p, ds, da, fv->status.p);
        check_launch();
    }
    mark(fv, "k_adjoint_nonowned", s);
    if (M.n_nonowned > 0) {
        k_adjoint_nonowned<DIM, NS, -1><<<blocks_for(M.n_nonowned, 128), 128, 0, s>>>(M, P, U, fv->adj_nb.p, rec, out, ds, da);
        check_launch();
    }
    mark(fv, "k_adjoint_gather", s);
    k_adjoint_gather<DIM, NS><<<blocks_for(M.n_cells, 128), 128, 0, s>>>(M, P, U, fv->aux.p, out, Ub, ds, da, fv->status.p);
    check_launch();
    mark(fv, "end", s);
}

}  // namespace abl
