// fv_adjoint.cuh -- reverse mode (vector-Jacobian product) of the FP64 RHS, sm_100a.
//
// Given a residual weight Fbar (one row per cell, read on owned cells), the VJP accumulates
// Ubar += (dF/dU)^T Fbar for every cell, boundary ghosts and halos included. It is the exact
// transpose of the tangent the dual-number kernels propagate (the derivative of the branch the primal
// evaluation takes at limiter minima, flux-splitting switches and mass-fraction clips).
//
// Of the forward pass only per-cell data is kept: the limited gradients and aux gradients one RHS
// keeps anyway, plus the unlimited gradient, the limiter factor and the minimising face per component.
// Every per-face intermediate (face states, EOS decode, flux calculator) is recomputed:
//   k_gradient          forward gradients, with the limiter records
//   k_tile_adjoint      one CTA per tile. Per face, colour by colour: recompute the face states, the
//                       EOS decode and the flux calculator, then run the flux backwards; the adjoint of
//                       each side's state, limited gradient, aux and aux gradient is summed into that
//                       cell's shared-memory accumulators (faces of one colour touch distinct cells, so
//                       no atomics and a fixed order). Then per tile cell the limiter and least-squares
//                       gradient are run backwards from the records of the forward gradient pass.
//   k_adjoint_nonowned  the same cell step for boundary ghosts and halos, from per-face records.
//   k_adjoint_gather    per cell: the neighbour terms of the gradient, limiter and aux-gradient adjoints
//                       (a gather over the cell's faces, the transpose of the forward gathers), then the
//                       aux (T, u, Y) chain rule, added into Ubar.
//
// Reference functions reversed: CellInterpolant::ComputeFieldGradients and the limiter
// (src/finiteVolume/cellInterpolant.cpp:282-497), ComputeFluxSourceTerms and ProjectToFace (:499-639,
// :890-950), NavierStokesTransport::AdvectionFlux / DiffusionFlux (navierStokesTransport.cpp:99-207,
// 454-532), SpeciesTransport fluxes (speciesTransport.cpp:112-341), the flux calculators
// (ausm.cpp:2-43, ausmpUp.cpp:5-96, riemann.cpp / riemannSolver.cpp), PerfectGas and TChem decode.
#pragma once
#include "fv_kernels.cuh"

namespace abl {

// ---------------------------------------------------------------------------------------------------
// EOS pieces
// ---------------------------------------------------------------------------------------------------
// e = U1/rho - |rho u|^2 / (2 rho^2)
template <int DIM>
ABL_HD void internal_energy_vjp(const double* U, double eb, double* Ub) {
    const double irho = rcp64(U[0]);
    double vu = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double vel = U[2 + d] * irho;
        Ub[2 + d] -= eb * vel * irho;
        vu += vel * U[2 + d];
    }
    Ub[1] += eb * irho;
    Ub[0] -= eb * (U[1] - vu) * irho * irho;
}

template <class S>
ABL_HD S nasa_dcp_molar(const double* c, S T) {
    const double* a = (T < c[0]) ? c + 1 : c + 8;
    return kRuniv * (a[1] + T * (2.0 * a[2] + T * (3.0 * a[3] + T * 4.0 * a[4])));
}

// reverse of fill_y (clip to [0, 1], renormalise or close with the last species)
template <int NSMAX>
ABL_HD void fill_y_vjp(int ns, double rho, const double* rhoY, const double* ysb, double* rhob, double* rhoYb) {
    const double irho = rcp64(rho);
    double y[NSMAX > 0 ? NSMAX : 1];
    bool act[NSMAX > 0 ? NSMAX : 1];
    double sum = 0.0;
ABL_UNROLL_SPECIES
    for (int s = 0; s < ns - 1; s++) {
        const double raw = rhoY[s] * irho;
        act[s] = raw > 0.0 && !(1.0 < raw);
        y[s] = pmin(1.0, pmax(0.0, raw));
        sum += y[s];
    }
    double irhob = 0.0, dot = 0.0;
    if (sum > 1.0) {
ABL_UNROLL_SPECIES
        for (int s = 0; s < ns - 1; s++) dot += ysb[s] * y[s];
    }
ABL_UNROLL_SPECIES
    for (int s = 0; s < ns - 1; s++) {
        double yb = sum > 1.0 ? ysb[s] / sum - dot / (sum * sum) : ysb[s] - ysb[ns - 1];
        if (!act[s]) yb = 0.0;
        rhoYb[s] += yb * irho;
        irhob += yb * rhoY[s];
    }
    *rhob -= irhob * irho * irho;
}

// reverse of the mixture temperature T(e_ref, Y) (implicit function of e_s(T, Y) = e_ref)
template <int DIM, int NSMAX>
ABL_HD void nasa_temperature_vjp(const Phys& P, int ns, const double* U, const double* ys, double T, double Tb, double* ysb, double* Ub) {
    double cv = 0;
ABL_UNROLL_SPECIES
    for (int k = 0; k < ns; k++) cv += ys[k] * (nasa_cp_molar(P.nasa7 + 15 * k, T) - kRuniv) * P.inv_mw[k];
    const double q = Tb / cv;
ABL_UNROLL_SPECIES
    for (int k = 0; k < ns; k++)
        ysb[k] -= q * (nasa_h_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] - P.href[k] - kRuniv * T * P.inv_mw[k]);
    internal_energy_vjp<DIM>(U, q, Ub);
}

// reverse of decode(): adjoints of the decoded e, a, p into the face state U
template <int DIM, int NSMAX>
ABL_HD void decode_vjp(const Phys& P, int ns, const double* U, const Decoded<double>& dd, double eb, double ab, double pb, double* Ub) {
    const double rho = U[0];
    if (NSMAX == 0 || P.eos == ABL_EOS_PERFECT_GAS) {
        const double cv = P.r_gas / (P.gamma - 1.0);
        double Tb = eb * cv + pb * P.r_gas * rho;
        if (dd.a > 0) Tb += ab * P.gamma * P.r_gas / (2.0 * dd.a);
        Ub[0] += pb * P.r_gas * dd.T;
        internal_energy_vjp<DIM>(U, Tb * rcp64(cv), Ub);
        return;
    }
    constexpr int NY = NSMAX > 0 ? NSMAX : 1;
    double ys[NY], ysb[NY];
    fill_y(ns, rho, U + 2 + DIM, ys);
    const double T = dd.T;
    double cp = 0, iw = 0, dcp = 0;
ABL_UNROLL_SPECIES
    for (int k = 0; k < ns; k++) {
        cp += ys[k] * nasa_cp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k];
        dcp += ys[k] * nasa_dcp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k];
        iw += ys[k] * P.inv_mw[k];
        ysb[k] = 0.0;
    }
    const double R = kRuniv * rcp64(rcp64(iw));
    const double cv = cp - R;
    const double gamma = cp * rcp64(cv);
    const double q = dd.a > 0 ? ab / (2.0 * dd.a) : 0.0;  // a = sqrt(gamma R T)
    const double gb = q * R * T;
    double Rb = q * gamma * T + pb * rho * T;
    double Tb = q * gamma * R + pb * rho * R;
    Ub[0] += pb * R * T;
    const double cpb = -gb * R / (cv * cv);
    Rb += gb * cp / (cv * cv);
    Tb += cpb * dcp;
    // e = e_s(T, Y): de/dT = cv, de/dY_k = e_s,k
ABL_UNROLL_SPECIES
    for (int k = 0; k < ns; k++) {
        const double esk = nasa_h_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] - P.href[k] - kRuniv * T * P.inv_mw[k];
        ysb[k] += eb * esk + cpb * nasa_cp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] + Rb * kRuniv * P.inv_mw[k];
    }
    Tb += eb * cv;
    nasa_temperature_vjp<DIM, NSMAX>(P, ns, U, ys, T, Tb, ysb, Ub);
    fill_y_vjp<NSMAX>(ns, rho, U + 2 + DIM, ysb, Ub, Ub + 2 + DIM);
}

// reverse of cp_at (conductivity of Sutherland / constant-Lewis transport)
template <int DIM, int NSMAX>
ABL_HD void cp_at_vjp(const Phys& P, int ns, const double* U, double T, double cpb, double* Ub, double* Tb) {
    if (NSMAX == 0 || P.eos == ABL_EOS_PERFECT_GAS) return;
    constexpr int NY = NSMAX > 0 ? NSMAX : 1;
    double ys[NY], ysb[NY];
    fill_y(ns, U[0], U + 2 + DIM, ys);
    double dcp = 0;
ABL_UNROLL_SPECIES
    for (int k = 0; k < ns; k++) {
        dcp += ys[k] * nasa_dcp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k];
        ysb[k] = cpb * nasa_cp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k];
    }
    *Tb += cpb * dcp;
    fill_y_vjp<NSMAX>(ns, U[0], U + 2 + DIM, ysb, Ub, Ub + 2 + DIM);
}

// reverse of transport(): adjoints of mu, k, D into the face state and the face temperature
template <int DIM, int NSMAX>
ABL_HD void transport_vjp(const Phys& P, int ns, const double* U, double T, double mub, double kb, double Db, double* Ub, double* Tb) {
    switch (P.transport) {
        case ABL_TRANSPORT_SUTHERLAND: {
            const double pr = 0.707, sc = 0.707, so = 111.0;
            const double m = sutherland_mu(T);
            const double cp = cp_at<DIM, NSMAX>(P, ns, U, T);
            const double mb = mub + kb * cp / pr + Db / (U[0] * sc);
            Ub[0] -= Db * m / (U[0] * U[0] * sc);
            *Tb += mb * m * (1.5 / T - 1.0 / (T + so));
            cp_at_vjp<DIM, NSMAX>(P, ns, U, T, kb * m / pr, Ub, Tb);
            return;
        }
        case ABL_TRANSPORT_CONSTANT_LEWIS: {
            const double cp = cp_at<DIM, NSMAX>(P, ns, U, T);
            const double k = P.mu * cp / P.k;
            const double D = k / (U[0] * cp * P.diff);
            const double kbt = kb + Db / (U[0] * cp * P.diff);
            Ub[0] -= Db * D / U[0];
            cp_at_vjp<DIM, NSMAX>(P, ns, U, T, kbt * P.mu / P.k - Db * D / cp, Ub, Tb);
            return;
        }
        default:
            return;  // constant properties
    }
}

// reverse of cell_aux(): aux = (T, u, Y) of a cell from its conserved state
template <int DIM, int NS>
__device__ __forceinline__ void cell_aux_vjp(const Phys& P, const double* u, const double* __restrict__ aux, int c, const double* ab, double* Ub) {
    using D = Dims<DIM, NS>;
    const double irho = rcp64(u[0]);
    double irhob = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        Ub[2 + d] += ab[1 + d] * irho;
        irhob += ab[1 + d] * u[2 + d];
    }
ABL_UNROLL_SPECIES
    for (int s = 0; s < NS; s++) {
        Ub[D::NE + s] += ab[1 + DIM + s] * irho;
        irhob += ab[1 + DIM + s] * u[D::NE + s];
    }
    Ub[0] -= irhob * irho * irho;
    if (ab[0] == 0.0) return;
    if (NS > 0 && P.eos == ABL_EOS_NASA7) {
        constexpr int NY = NS > 0 ? NS : 1;
        double ys[NY], ysb[NY];
        fill_y(NS, u[0], u + D::NE, ys);
        bool ok = true;
        const double T = temperature<DIM, NS>(P, NS, u, __ldg(aux + (size_t)c * D::NA), &ok);
ABL_UNROLL_SPECIES
        for (int k = 0; k < NS; k++) ysb[k] = 0.0;
        nasa_temperature_vjp<DIM, NS>(P, NS, u, ys, T, ab[0], ysb, Ub);
        fill_y_vjp<NS>(NS, u[0], u + D::NE, ysb, Ub, Ub + D::NE);
    } else {
        internal_energy_vjp<DIM>(u, ab[0] * rcp64(P.r_gas / (P.gamma - 1.0)), Ub);
    }
}

// ---------------------------------------------------------------------------------------------------
// flux calculators: g[0..7] += d(mf, p12)/d(uL, aL, rhoL, pL, uR, aR, rhoR, pR)^T (mfb, p12b)
// ---------------------------------------------------------------------------------------------------
ABL_HD double sgn1(double m) { return m < 0 ? -1.0 : 1.0; }  // the derivative of dabs()

ABL_HD void ausm_vjp(const double* x, double mfb, double p12b, double* g) {
    const double uL = x[0], aL = x[1], rhoL = x[2], pL = x[3], uR = x[4], aR = x[5], rhoR = x[6], pR = x[7];
    const double iaR = rcp64(aR), iaL = rcp64(aL);
    const double Mm = uR * iaR, Mp = uL * iaL;
    const bool inM = fabs(Mm) <= 1.0, inP = fabs(Mp) <= 1.0;
    double sMm, sPm, sMp, sPp;
    if (inM) {
        sMm = -0.25 * sqr(Mm - 1.0);
        sPm = -sMm * (2.0 + Mm);
    } else {
        sMm = 0.5 * (Mm - fabs(Mm));
        sPm = sMm / Mm;
    }
    if (inP) {
        sMp = 0.25 * sqr(Mp + 1.0);
        sPp = sMp * (2.0 - Mp);
    } else {
        sMp = 0.5 * (Mp + fabs(Mp));
        sPp = sMp / Mp;
    }
    const double m = sMm + sMp;
    const double sPmb = p12b * pR, sPpb = p12b * pL;
    g[7] += p12b * sPm;
    g[3] += p12b * sPp;
    double mb;
    if (m < 0) {
        mb = mfb * aR * rhoR;
        g[5] += mfb * m * rhoR;
        g[6] += mfb * m * aR;
    } else {
        mb = mfb * aL * rhoL;
        g[1] += mfb * m * rhoL;
        g[2] += mfb * m * aL;
    }
    double sMmb = mb, sMpb = mb, Mmb = 0, Mpb = 0;
    if (inM) {
        sMmb -= sPmb * (2.0 + Mm);
        Mmb -= sPmb * sMm;
        Mmb -= sMmb * 0.5 * (Mm - 1.0);
    } else {
        sMmb += sPmb / Mm;
        Mmb -= sPmb * sPm / Mm;
        Mmb += sMmb * 0.5 * (1.0 - sgn1(Mm));
    }
    if (inP) {
        sMpb += sPpb * (2.0 - Mp);
        Mpb -= sPpb * sMp;
        Mpb += sMpb * 0.5 * (Mp + 1.0);
    } else {
        sMpb += sPpb / Mp;
        Mpb -= sPpb * sPp / Mp;
        Mpb += sMpb * 0.5 * (1.0 + sgn1(Mp));
    }
    g[4] += Mmb * iaR;
    g[5] -= Mmb * Mm * iaR;
    g[0] += Mpb * iaL;
    g[1] -= Mpb * Mp * iaL;
}

// derivatives of the AUSM+up splitting polynomials (Ausmpup in fv_physics.cuh)
struct AusmpupD {
    static ABL_HD double M2P(double m) { return 0.25 * sqr(m + 1.0); }
    static ABL_HD double M2M(double m) { return -0.25 * sqr(m - 1.0); }
    static ABL_HD double dM2P(double m) { return 0.5 * (m + 1.0); }
    static ABL_HD double dM2M(double m) { return -0.5 * (m - 1.0); }
    static ABL_HD double dM4P(double m) {
        if (fabs(m) >= 1.0) return 0.5 * (1.0 + sgn1(m));
        return dM2P(m) * (1.0 - 2.0 * M2M(m)) - 2.0 * M2P(m) * dM2M(m);
    }
    static ABL_HD double dM4M(double m) {
        if (fabs(m) >= 1.0) return 0.5 * (1.0 - sgn1(m));
        return dM2M(m) * (1.0 + 2.0 * M2P(m)) + 2.0 * M2M(m) * dM2P(m);
    }
    // d/dm and d/dfa of P5P, P5M
    static ABL_HD void dP5P(double m, double fa, double* dm, double* dfa) {
        if (fabs(m) >= 1.0) {
            const double e = m + 1E-30, m1 = 0.5 * (m + fabs(m));
            *dm = (0.5 * (1.0 + sgn1(m)) * e - m1) / (e * e);
            *dfa = 0.0;
            return;
        }
        const double al = 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa);
        const double B = (2.0 - m) - 16.0 * al * m * M2M(m);
        *dm = dM2P(m) * B + M2P(m) * (-1.0 - 16.0 * al * (M2M(m) + m * dM2M(m)));
        *dfa = -30.0 * fa * m * M2P(m) * M2M(m);
    }
    static ABL_HD void dP5M(double m, double fa, double* dm, double* dfa) {
        if (fabs(m) >= 1.0) {
            const double e = m + 1E-30, m1 = 0.5 * (m - fabs(m));
            *dm = (0.5 * (1.0 - sgn1(m)) * e - m1) / (e * e);
            *dfa = 0.0;
            return;
        }
        const double al = 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa);
        const double B = (-2.0 - m) + 16.0 * al * m * M2P(m);
        *dm = dM2M(m) * B + M2M(m) * (-1.0 + 16.0 * al * (M2P(m) + m * dM2P(m)));
        *dfa = 30.0 * fa * m * M2M(m) * M2P(m);
    }
};

ABL_HD void ausmpup_vjp(double mInf, double alpha, const double* x, double mfb, double p12b, double* g) {
    using A = Ausmpup<double>;
    using B = AusmpupD;
    const double uL = x[0], aL = x[1], rhoL = x[2], pL = x[3], uR = x[4], aR = x[5], rhoR = x[6], pR = x[7];
    const double Kp = 0.25, Ku = 0.75, sigma = 0.25;
    // forward
    const double rho12 = 0.5 * (rhoL + rhoR);
    const double ialpha = rcp64(alpha);
    const double a12 = 0.5 * (aL + aR) * ialpha;
    const double ia12 = rcp64(a12);
    const double mL = uL * ia12, mR = uR * ia12;
    const double mBar2 = (sqr(uL) + sqr(uR)) * (0.5 * ia12 * ia12);
    double fa = 1.0, mO = 0.0, xmax = 0.0;
    const double mInf2 = sqr(mInf);
    if (mInf > 0) {
        xmax = pmax(mBar2, mInf2);
        mO = sqrt(pmin(1.0, xmax));
        fa = mO * (2.0 - mO);
    }
    const double a2 = alpha * alpha;
    const double c = Kp * rcp64(fa);
    const double w1 = 1.0 - sigma * mBar2;
    const double w = pmax(w1, 0.0);
    const double dp = pR - pL;
    const double den = rho12 * a12 * a12 * a2;
    const double idn = rcp64(den);
    const double m12 = A::M4P(mL) + A::M4M(mR) - c * w * dp * idn;
    const double p5P = A::P5P(mL, fa), p5M = A::P5M(mR, fa);
    // reverse
    double mLb = 0, mRb = 0, fab = 0, a12b = 0, rho12b = 0, mBar2b = 0;
    const double vb = p12b * rcp64(sqr(alpha));
    g[3] += vb * p5P;
    g[7] += vb * p5M;
    const double K = Ku * rho12 * fa * a12 * a12 * a2 * (mR - mL);
    const double p5Pb = vb * (pL - p5M * K), p5Mb = vb * (pR - p5P * K);
    const double Q = -vb * Ku * p5P * p5M * a2;
    rho12b += Q * fa * a12 * a12 * (mR - mL);
    fab += Q * rho12 * a12 * a12 * (mR - mL);
    a12b += Q * rho12 * fa * 2.0 * a12 * (mR - mL);
    mRb += Q * rho12 * fa * a12 * a12;
    mLb -= Q * rho12 * fa * a12 * a12;
    double dm, dfa;
    B::dP5P(mL, fa, &dm, &dfa);
    mLb += p5Pb * dm;
    fab += p5Pb * dfa;
    B::dP5M(mR, fa, &dm, &dfa);
    mRb += p5Mb * dm;
    fab += p5Mb * dfa;
    double m12b;
    if (m12 > 0) {
        m12b = mfb * a12 * rhoL;
        a12b += mfb * m12 * rhoL;
        g[2] += mfb * a12 * m12;
    } else {
        m12b = mfb * a12 * rhoR;
        a12b += mfb * m12 * rhoR;
        g[6] += mfb * a12 * m12;
    }
    mLb += m12b * B::dM4P(mL);
    mRb += m12b * B::dM4M(mR);
    const double tb = -m12b;
    const double cb = tb * w * dp * idn, wb = tb * c * dp * idn, dpb = tb * c * w * idn, idnb = tb * c * w * dp;
    const double denb = -idnb * idn * idn;
    fab -= cb * Kp / (fa * fa);
    if (!(w1 < 0.0)) mBar2b -= sigma * wb;
    g[7] += dpb;
    g[3] -= dpb;
    rho12b += denb * a12 * a12 * a2;
    a12b += denb * rho12 * 2.0 * a12 * a2;
    if (mInf > 0) {
        const double mOb = fab * (2.0 - 2.0 * mO);
        const double mO2b = mO > 0 ? mOb / (2.0 * mO) : 0.0;
        if (!(1.0 < xmax) && !(mBar2 < mInf2)) mBar2b += mO2b;
    }
    double ia12b = mBar2b * (sqr(uL) + sqr(uR)) * ia12;
    g[0] += mBar2b * uL * ia12 * ia12 + mLb * ia12;
    g[4] += mBar2b * uR * ia12 * ia12 + mRb * ia12;
    ia12b += mLb * uL + mRb * uR;
    a12b -= ia12b * ia12 * ia12;
    g[1] += 0.5 * a12b * ialpha;
    g[5] += 0.5 * a12b * ialpha;
    g[2] += 0.5 * rho12b;
    g[6] += 0.5 * rho12b;
}

// any calculator: eight tangent evaluations (exact Riemann, average)
ABL_HD void calc_vjp_tangents(const Phys& P, const double* x, double mfb, double p12b, double* g, bool* rok) {
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
        Dual xi[8];
#pragma unroll
        for (int j = 0; j < 8; j++) xi[j] = Dual(x[j], i == j ? 1.0 : 0.0);
        Dual mf, p12;
        flux_calc<Dual>(P, xi[0], xi[1], xi[2], xi[3], xi[4], xi[5], xi[6], xi[7], &mf, &p12, rok);
        g[i] += mfb * mf.d + p12b * p12.d;
    }
}

template <int FK>
ABL_HD void calc_vjp(const Phys& P, const double* x, double mfb, double p12b, double* g, bool* rok) {
    const int kind = FK >= 0 ? FK : P.flux;
    if (kind == ABL_FLUX_AUSM)
        ausm_vjp(x, mfb, p12b, g);
    else if (kind == ABL_FLUX_AUSMPUP)
        ausmpup_vjp(P.minf, P.alpha, x, mfb, p12b, g);
    else
        calc_vjp_tangents(P, x, mfb, p12b, g, rok);
}

// ---------------------------------------------------------------------------------------------------
// face fluxes backwards
// ---------------------------------------------------------------------------------------------------
// Two lanes per face: lanes 2j (left side) and 2j+1 (right side) of a warp hold one face. Each lane
// projects, decodes and reverses its own side; what couples the sides (the flux calculator and the
// upwind choice, the averaged face state of the diffusion flux) is exchanged with the partner lane and
// evaluated identically in both. Every exchange sits in control flow both lanes take.
__device__ __forceinline__ double xch(unsigned mask, double v) { return __shfl_xor_sync(mask, v, 1); }

// advection (NavierStokesTransport::AdvectionFlux + SpeciesTransport::AdvectionFlux) backwards for
// this lane's side: fb = flux adjoint, ub += adjoint of this side's projected face state u
template <int DIM, int NS, int FK>
__device__ __forceinline__ void advection_vjp_side(const Phys& P, unsigned mask, int side, const double* normal, const double* u, double Tguess,
                                                   bool adv, bool spadv, const double* fb, double* ub, bool* ok, bool* rok) {
    using D = Dims<DIM, NS>;
    double areaMag = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) areaMag += normal[d] * normal[d];
    areaMag = sqrt(areaMag);
    const double iA = rcp64(areaMag);
    double norm[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) norm[d] = normal[d] * iA;
    const auto dd = decode<DIM, NS>(P, NS, u, Tguess, ok);
    const double rho = u[0], irho = rcp64(rho);
    double vel[DIM], un = 0, v2 = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = u[2 + d] * irho;
        un += vel[d] * norm[d];
        v2 += vel[d] * vel[d];
    }
    const double vm = sqrt(v2);
    const double H = dd.e + vm * vm / 2.0 + dd.p * irho;
    // the flux calculator on both sides' values, in (left, right) order in both lanes
    const double un_o = xch(mask, un), a_o = xch(mask, dd.a), rho_o = xch(mask, rho), p_o = xch(mask, dd.p);
    const double x[8] = {side ? un_o : un, side ? a_o : dd.a, side ? rho_o : rho, side ? p_o : dd.p,
                         side ? un : un_o, side ? dd.a : a_o, side ? rho : rho_o, side ? dd.p : p_o};
    double mf, p12;
    const int dir = flux_calc_k<FK, double>(P, x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], &mf, &p12, rok);
    const double mA = mf * areaMag;
    const double H_o = xch(mask, H);
    double vel_o[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) vel_o[d] = xch(mask, vel[d]);
    // LEFT upwinds side 0, RIGHT side 1; for the species anything but LEFT takes side 1
    const bool upme = (dir == ABL_DIR_LEFT) == (side == 0);
    double mfb = 0, p12b = 0, eb = 0, pb = 0, irhob = 0, velb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) velb[d] = 0.0;
    if (adv) {
        mfb += areaMag * fb[0];
#pragma unroll
        for (int n = 0; n < DIM; n++) p12b += normal[n] * fb[2 + n];
        if (dir == ABL_DIR_LEFT || dir == ABL_DIR_RIGHT) {
            double sacc = (upme ? H : H_o) * fb[1];
#pragma unroll
            for (int n = 0; n < DIM; n++) sacc += (upme ? vel[n] : vel_o[n]) * fb[2 + n];
            mfb += areaMag * sacc;
            if (upme) {
                const double Hb = mA * fb[1];
                eb += Hb;
                pb += Hb * irho;
                irhob += Hb * dd.p;
#pragma unroll
                for (int n = 0; n < DIM; n++) velb[n] += Hb * vel[n] + mA * fb[2 + n];
            }
        } else {
            double sacc = 0.5 * (H + H_o) * fb[1];
#pragma unroll
            for (int n = 0; n < DIM; n++) sacc += 0.5 * (vel[n] + vel_o[n]) * fb[2 + n];
            mfb += areaMag * sacc;
            const double Hb = 0.5 * mA * fb[1];
            eb += Hb;
            pb += Hb * irho;
            irhob += Hb * dd.p;
#pragma unroll
            for (int n = 0; n < DIM; n++) velb[n] += Hb * vel[n] + 0.5 * mA * fb[2 + n];
        }
    }
    if (NS > 0 && spadv && dir == ABL_DIR_NA && P.sp_compact) {
        // compact process, no direction: flux_s = mA (rhoY_L + rhoY_R) / (rho_L + rho_R) (both halves)
        const double rhoM = 0.5 * (rho + rho_o), irm = 1.0 / rhoM;
ABL_UNROLL_SPECIES
        for (int s = 0; s < NS; s++) {
            const double ry = u[D::NE + s], ry_o = xch(mask, ry);
            const double num = 0.5 * (side ? ry + ry_o : ry_o + ry);
            mfb += areaMag * num * irm * fb[D::NE + s];
            ub[D::NE + s] += 0.5 * mA * irm * fb[D::NE + s];
            ub[0] -= 0.5 * mA * num * irm * irm * fb[D::NE + s];
        }
    } else if (NS > 0 && spadv) {
ABL_UNROLL_SPECIES
        for (int s = 0; s < NS; s++) {
            const double Y = u[D::NE + s] * irho;
            const double Y_o = xch(mask, Y);
            mfb += areaMag * (upme ? Y : Y_o) * fb[D::NE + s];
            if (upme) {
                const double Yb = mA * fb[D::NE + s];
                ub[D::NE + s] += Yb * irho;
                irhob += Yb * u[D::NE + s];
            }
        }
    }
    double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (mfb != 0.0 || p12b != 0.0) calc_vjp<FK>(P, x, mfb, p12b, g, rok);
    const double gu = side ? g[4] : g[0], ga = side ? g[5] : g[1], gr = side ? g[6] : g[2], gp = side ? g[7] : g[3];
    ub[0] += gr;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        velb[d] += gu * norm[d];
        ub[2 + d] += velb[d] * irho;
        irhob += velb[d] * u[2 + d];
    }
    ub[0] -= irhob * irho * irho;
    decode_vjp<DIM, NS>(P, NS, u, dd, eb, ga, pb + gp, ub);
}

// diffusion (NavierStokesTransport::DiffusionFlux, SpeciesTransport diffusion) backwards. fs, fa and
// gf are the face state, aux and aux gradient (averages of the two cells); each side receives half of
// the returned fsb, fab, gfb.
template <int DIM, int NS>
__device__ __forceinline__ void diffusion_vjp(const Phys& P, const double* normal, const double* fs, const double* fa, const double* gf, bool dif,
                                              bool spdif, const double* fb, double* fsb, double* fab, double* gfb) {
    using D = Dims<DIM, NS>;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) fsb[k] = 0.0;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA; k++) fab[k] = 0.0;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA * DIM; k++) gfb[k] = 0.0;
    double mu, kc, diff;
    transport<DIM, NS>(P, NS, fs, fa[0], &mu, &kc, &diff);
    double mub = 0, kb = 0, Db = 0;
    if (dif) {
        const double* gT = gf;
        const double* gv = gf + DIM;
        double divVel = 0;
#pragma unroll
        for (int c = 0; c < DIM; ++c) divVel += gv[c * DIM + c];
        double tau[DIM * DIM], taub[DIM * DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                tau[c * DIM + d] = (d == c) ? 2.0 * mu * (gv[c * DIM + d] - divVel / 3.0) : mu * (gv[c * DIM + d] + gv[d * DIM + c]);
                taub[c * DIM + d] = -normal[d] * fb[2 + c];
            }
        // energy: -sum_d n_d (sum_c u_c tau_dc + k dT/dx_d)
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                taub[d * DIM + c] -= normal[d] * fa[1 + c] * fb[1];
                fab[1 + c] -= normal[d] * tau[d * DIM + c] * fb[1];
            }
            kb -= normal[d] * gT[d] * fb[1];
            gfb[d] -= normal[d] * kc * fb[1];
        }
        double divb = 0;
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double tb = taub[c * DIM + d];
                if (c == d) {
                    gfb[DIM + c * DIM + c] += 2.0 * mu * tb;
                    divb -= 2.0 * mu / 3.0 * tb;
                    mub += 2.0 * tb * (gv[c * DIM + c] - divVel / 3.0);
                } else {
                    gfb[DIM + c * DIM + d] += mu * tb;
                    gfb[DIM + d * DIM + c] += mu * tb;
                    mub += tb * (gv[c * DIM + d] + gv[d * DIM + c]);
                }
            }
#pragma unroll
        for (int c = 0; c < DIM; ++c) gfb[DIM + c * DIM + c] += divb;
    }
    if constexpr (NS > 0) {
        if (spdif) {
            const double density = fs[0];
            const int yoff = (1 + DIM) * DIM;
            double rhob = 0, Tb = 0;
ABL_UNROLL_SPECIES
            for (int s = 0; s < NS; ++s) {
                const double hs = P.eos == ABL_EOS_NASA7 ? nasa_h_molar(P.nasa7 + 15 * s, fa[0]) * P.inv_mw[s] - P.href[s] : 0.0;
                // one constant D_k per species (no state dependence), or the transport model's D
                const double Ds = P.diff_k ? P.diff_k[s] : diff;
                double hsb = 0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double gy = gf[yoff + s * DIM + d];
                    const double q = -normal[d] * (fb[D::NE + s] + hs * fb[1]);
                    rhob += q * Ds * gy;
                    if (!P.diff_k) Db += q * density * gy;
                    gfb[yoff + s * DIM + d] += q * density * Ds;
                    hsb -= normal[d] * density * Ds * gy * fb[1];
                }
                if (P.eos == ABL_EOS_NASA7) Tb += hsb * nasa_cp_molar(P.nasa7 + 15 * s, fa[0]) * P.inv_mw[s];
            }
            fsb[0] += rhob;
            fab[0] += Tb;
        }
    }
    transport_vjp<DIM, NS>(P, NS, fs, fa[0], mub, kb, Db, fsb, &fab[0]);
}

// ---------------------------------------------------------------------------------------------------
// per-cell accumulators: [state NC][limited gradient NC*DIM][aux NA][aux gradient NA*DIM]
template <int DIM, int NS>
struct AdjRow {
    using D = Dims<DIM, NS>;
    static constexpr int U = 0, G = D::NC, A = D::NC + D::NC * DIM, GA = D::NC + D::NC * DIM + D::NA;
    static constexpr int N = GA + D::NA * DIM;
    static constexpr int S = N | 1;  // shared-memory row stride: odd, so rows of random cells spread over the banks
};

// one face backwards, this lane's side: the adjoint contributions are added into the side's
// accumulator row dst (nullptr drops a side that another tile accumulates)
template <int DIM, int NS, int FK>
__device__ __forceinline__ void face_vjp_side(const DevMesh& M, const Phys& P, unsigned mask, int side, int me, const double* normal,
                                              const double* fdxo, const double* __restrict__ U, const double* __restrict__ aux,
                                              const double* __restrict__ grad, const double* __restrict__ agrad, const double* __restrict__ Fb,
                                              double* dst, bool* ok, bool* rok) {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, double>;
    using AR = AdjRow<DIM, NS>;
    // dF_L/dflux = -1/V_L, dF_R/dflux = +1/V_R on owned cells; fb = (right term) + (left term)
    const bool own = M.kind[me] == ABL_CELL_OWNED;
    const double iv = own ? M.ivol[me] : 0.0;
    double fb[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        const double t = own ? __ldg(Fb + (size_t)me * D::NC + k) * iv : 0.0;
        const double mine = side ? t : -t;
        fb[k] = mine + xch(mask, mine);
    }
    double c[D::NC];
    load_state<DIM, NS>(U, me, c);
    const bool adv = P.advection && P.flux != ABL_FLUX_OFF;
    const bool spadv = NS > 0 && P.sp_adv && P.flux != ABL_FLUX_OFF;
    if (adv || spadv) {
        const bool lsq = P.recon == ABL_RECON_LEASTSQUARES;
        double u[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            double dot = 0;
            if (lsq) {
#pragma unroll
                for (int d = 0; d < DIM; d++) dot += __ldg(grad + (size_t)me * GR::GS + k * DIM + d) * fdxo[d];
            }
            u[k] = lsq ? c[k] + dot : c[k];
        }
        double guess = 300.0;
        if (NS > 0 && P.eos == ABL_EOS_NASA7) {
            const double Tme = __ldg(aux + (size_t)me * D::NA), To = xch(mask, Tme);
            const double TL = side ? To : Tme, TR = side ? Tme : To;
            guess = side ? TL * .33 + .67 * TR : TL * .67 + .33 * TR;
        }
        double ub[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) ub[k] = 0.0;
        advection_vjp_side<DIM, NS, FK>(P, mask, side, normal, u, guess, adv, spadv, fb, ub, ok, rok);
        // u_face = u_cell + g . dx: the identity part to the state, the outer product with dx to the gradient
        if (dst) {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) {
                dst[AR::U + k] += ub[k];
                if (lsq)
#pragma unroll
                    for (int d = 0; d < DIM; d++) dst[AR::G + k * DIM + d] += ub[k] * fdxo[d];
            }
        }
    }
    const bool dif = P.diffusion && P.transport != ABL_TRANSPORT_NONE;
    const bool spdif = NS > 0 && P.sp_dif && P.transport != ABL_TRANSPORT_NONE;
    if (dif || spdif) {
        // face averages: a + b is commutative, so both lanes hold identical values
        double fs[D::NC], fa[D::NA], gf[D::NA * DIM];
        {
            double a[D::NA];
            cell_aux<DIM, NS>(P, c, aux, me, a);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) fa[k] = a[k] * 0.5 + xch(mask, a[k]) * 0.5;
        }
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) fs[k] = c[k] * 0.5 + xch(mask, c[k]) * 0.5;
        // the face gradient: in 1D the two-cell LeastSquares stencil's (w_L a_L + w_R a_R, the same sum
        // in both lanes), else the average of the two cells' aux gradients
        double wme = 0.0;
        if constexpr (DIM == 1) {
            const double xme = fdxo[0], xot = xch(mask, fdxo[0]);  // each lane holds its side's offset
            const double fdx2[6] = {side ? xot : xme, 0.0, 0.0, side ? xme : xot, 0.0, 0.0};
            double wl, wr;
            face_weights_1d(fdx2, &wl, &wr);
            wme = side ? wr : wl;
            const double wot = side ? wl : wr;
            double a[D::NA];
            cell_aux<DIM, NS>(P, c, aux, me, a);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) {
                const double mine = a[k] * wme, other = xch(mask, a[k]) * wot;
                gf[k] = side ? other + mine : mine + other;
            }
        } else {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA * DIM; k++) {
                const double gm = __ldg(agrad + (size_t)me * GR::AS + k);
                gf[k] = 0.5 * gm + 0.5 * xch(mask, gm);
            }
        }
        double fsb[D::NC], fab[D::NA], gfb[D::NA * DIM];
        diffusion_vjp<DIM, NS>(P, normal, fs, fa, gf, dif, spdif, fb, fsb, fab, gfb);
        if (dst) {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) dst[AR::U + k] += 0.5 * fsb[k];
            if constexpr (DIM == 1) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NA; k++) dst[AR::A + k] += 0.5 * fab[k] + wme * gfb[k];
            } else {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NA; k++) dst[AR::A + k] += 0.5 * fab[k];
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NA * DIM; k++) dst[AR::GA + k] += 0.5 * gfb[k];
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------
// cell step: limiter and least-squares gradient backwards (the limiter recomputed), aux-gradient self
// term; writes the per-cell records the gather reads
template <int DIM, int NS>
struct AdjOut {
    double* gb;     // [nc][GS] adjoint of the unlimited state gradient
    double* beta;   // [nc][NC] limiter term for the minimising neighbour
    int* fstar;     // [nc][NC] face of that neighbour, -1 for none
    double* gab;    // [nc][AS] adjoint of the aux gradient
    double* ub;     // [nc][NC] state adjoint, own terms
    double* ab;     // [nc][NA] aux adjoint, own terms
};

// forward records of k_gradient<..., REC = true>: unlimited gradient, applied limiter factor, and the
// cone entry of the minimising face per component
struct GradRec {
    const double* graw;
    const double* phi;
    const int* ist;
};

template <int DIM, int NS, int LIM>
__device__ __forceinline__ void cell_vjp(const DevMesh& M, const Phys& P, int c, const double* __restrict__ U, const double* acc,
                                         const GradRec& rec, const AdjOut<DIM, NS>& out, bool do_state, bool do_aux) {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, double>;
    using AR = AdjRow<DIM, NS>;
    const uint8_t kind = M.kind[c];
    double ub[D::NC], gbar[D::NC * DIM], beta[D::NC];
    int fst[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        ub[k] = acc[AR::U + k];
        beta[k] = 0.0;
        fst[k] = -1;
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC * DIM; k++) gbar[k] = 0.0;
    if (do_state && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO)) {
        // g~ = phi g (0 when cancelled): g-bar = phi g~-bar, plus the limiter's own dependence on g and on
        // the minimising neighbour through r = (u_n - u_c) / (2 g . dx)
        const double* g = rec.graw + (size_t)c * GR::GS;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            const double ph = __ldg(rec.phi + (size_t)c * D::NC + k);
            const int i = __ldg(rec.ist + (size_t)c * D::NC + k);
            double phib = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const double gt = acc[AR::G + k * DIM + d];
                gbar[k * DIM + d] = ph * gt;
                phib += gt * __ldg(g + k * DIM + d);
            }
            if (i < 0 || phib == 0.0) continue;
            const int2 ce = M.cone[i];
            const int f = ce.x, n = ce.y & kConeNbr, sc = (ce.y & kConeSide) ? 1 : 0;
            double v[DIM], denom = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                v[d] = __ldg(M.fdx + 6 * (size_t)f + 3 * sc + d) - __ldg(M.fdx + 6 * (size_t)f + 3 * (1 - sc) + d);
                denom += __ldg(g + k * DIM + d) * v[d];
            }
            const double idn = rcp64(denom);
            const double r = 0.5 * (__ldg(U + (size_t)n * D::NC + k) - __ldg(U + (size_t)c * D::NC + k)) * idn;
            const double dl = limiter_k<LIM, Dual>(P.limiter, Dual(r, 1.0)).d;
            const double rb = dl * phib;
            if (rb == 0.0 || !isfinite(rb) || !isfinite(r)) continue;
            const double bk = 0.5 * rb * idn;  // d r / d (u_n - u_c) = 1 / (2 denom)
            beta[k] = bk;
            fst[k] = f;
            ub[k] -= bk;
#pragma unroll
            for (int d = 0; d < DIM; d++) gbar[k * DIM + d] -= r * rb * idn * v[d];  // d r / d denom = -r / denom
        }
        // g = sum_f w_f (u_n - u_c): the own-cell term, with the cell's summed weights
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const double ws = __ldg(M.wsum + 6 * (size_t)c + d);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) ub[k] -= ws * gbar[k * DIM + d];
        }
    }
    double ab[D::NA], gab[D::NA * DIM];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA; k++) ab[k] = acc[AR::A + k];
    const bool auxg = do_aux && kind != ABL_CELL_HALO_OUTER;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA * DIM; k++) gab[k] = auxg ? acc[AR::GA + k] : 0.0;
    if (auxg) {
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const double ws = __ldg(M.wsum + 6 * (size_t)c + 3 + d);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) ab[k] -= ws * gab[k * DIM + d];
        }
    }
    if (out.gb) {
        double* o = out.gb + (size_t)c * GR::GS;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC * DIM; k++) o[k] = gbar[k];
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        out.beta[(size_t)c * D::NC + k] = beta[k];
        out.fstar[(size_t)c * D::NC + k] = fst[k];
        out.ub[(size_t)c * D::NC + k] = ub[k];
    }
    if (out.gab) {
        double* o = out.gab + (size_t)c * GR::AS;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NA * DIM; k++) o[k] = gab[k];
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA; k++) out.ab[(size_t)c * D::NA + k] = ab[k];
}

// ---------------------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------------------
// resident CTAs per SM the register budget targets (shared memory holds 2 tiles of accumulators at
// 0 species; one at the species counts)
template <int NS>
struct AdjBlocks {
    static constexpr int tile = NS == 0 ? 2 : 1;
};

// 256 threads: two lanes per face, one colour (at most 128 faces) per pass
template <int DIM, int NS, int FK, int LIM>
__global__ void __launch_bounds__(256, AdjBlocks<NS>::tile) k_tile_adjoint(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                                          const double* __restrict__ grad, const double* __restrict__ agrad,
                                                                          const double* __restrict__ Fb, GradRec rec, AdjOut<DIM, NS> out,
                                                                          double* __restrict__ nbrec, int do_state, int do_aux, int* status) {
    using AR = AdjRow<DIM, NS>;
    extern __shared__ double sacc[];  // [tile cells][AR::S]
    const int t = blockIdx.x;
    const int cb = M.tile_cell_ptr[t], nct = M.tile_cell_ptr[t + 1] - cb;
    for (int i = threadIdx.x; i < nct * AR::S; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    bool ok = true, rok = true;
    const int side = threadIdx.x & 1, pair = threadIdx.x >> 1;
    const int base = M.col_base[t], ncol = M.col_base[t + 1] - base - 1;
    const int fb = M.tile_face_ptr[t];
    for (int q = 0; q < ncol; q++) {
        const int qa = M.col_start[base + q] + pair;
        const bool act = qa < M.col_start[base + q + 1];
        const unsigned mask = __ballot_sync(0xffffffffu, act);  // both lanes of a face share act
        if (act) {
            const int i = fb + M.tf_adj[qa];  // the face record
            const int2 lr = M.tf_cells[i];
            const int me = side ? lr.y : lr.x;
            double normal[DIM], fdxo[3];
            const double* geo = M.tf_geo + 10 * geo_record(M, i);
#pragma unroll
            for (int d = 0; d < DIM; d++) normal[d] = __ldg(geo + d);
#pragma unroll
            for (int d = 0; d < 3; d++) fdxo[d] = __ldg(geo + 3 + 3 * side + d);
            // destination: this tile's accumulator, the record of a non-owned side, or none
            const uint32_t slots = M.tf_slot[i];
            const int slot = side ? int(slots >> 16) : int(slots & 0xffff);
            const int nb = M.tf_nb[i];
            double* dst = nullptr;
            if (slot != 0xffff)
                dst = sacc + (size_t)slot * AR::S;
            else if (nb >= 0 && M.kind[me] != ABL_CELL_OWNED)
                dst = nbrec + (size_t)nb * AR::N;
            face_vjp_side<DIM, NS, FK>(M, P, mask, side, me, normal, fdxo, U, aux, grad, agrad, Fb, dst, &ok, &rok);
        }
        __syncthreads();
    }
    for (int j = threadIdx.x; j < nct; j += blockDim.x)
        cell_vjp<DIM, NS, LIM>(M, P, M.tile_cells[cb + j], U, sacc + (size_t)j * AR::S, rec, out, do_state, do_aux);
    if (!ok) atomicOr(status, kStatusEos);
    if (!rok) atomicOr(status, kStatusRiemann);
}

template <int DIM, int NS, int LIM>
__global__ void __launch_bounds__(128) k_adjoint_nonowned(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ nbrec,
                                                          GradRec rec, AdjOut<DIM, NS> out, int do_state, int do_aux) {
    using AR = AdjRow<DIM, NS>;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M.n_nonowned) return;
    const int c = M.nonowned[j];
    double acc[AR::N];
ABL_UNROLL_SPECIES
    for (int k = 0; k < AR::N; k++) acc[k] = 0.0;
    for (int i = M.cone_ptr[c]; i < M.cone_ptr[c + 1]; i++) {
        const int nb = M.face_nb[M.cone[i].x];
        if (nb < 0) continue;
        const double* r = nbrec + (size_t)nb * AR::N;
ABL_UNROLL_SPECIES
        for (int k = 0; k < AR::N; k++) acc[k] += r[k];
    }
    cell_vjp<DIM, NS, LIM>(M, P, c, U, acc, rec, out, do_state, do_aux);
}

template <int DIM, int NS>
__global__ void __launch_bounds__(128) k_adjoint_gather(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                        AdjOut<DIM, NS> in, double* __restrict__ Ub, int do_state, int do_aux, int* status) {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, double>;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M.n_cells) return;
    double ub[D::NC], ab[D::NA];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) ub[k] = in.ub[(size_t)m * D::NC + k];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA; k++) ab[k] = in.ab[(size_t)m * D::NA + k];
    const int beg = M.cone_ptr[m];
    const size_t wb = weight_base(M, m, beg);
#pragma unroll 1
    for (int i = beg; i < M.cone_ptr[m + 1]; i++) {
        const int2 ce = M.cone[i];
        const int f = ce.x, n = ce.y & kConeNbr;
        double w[DIM], wa[DIM];
        cone_weights<DIM, double>(M.cwar, nullptr, wb + (size_t)(i - beg), w, wa);
        if (do_state) {
            if (!(ce.y & kConeBoundary)) {
                double gn[D::NC * DIM];
                load_row<D::NC * DIM, double>(in.gb + (size_t)n * GR::GS, gn);
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++)
#pragma unroll
                    for (int d = 0; d < DIM; d++) ub[k] += w[d] * gn[k * DIM + d];
            }
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++)
                if (__ldg(in.fstar + (size_t)n * D::NC + k) == f) ub[k] += __ldg(in.beta + (size_t)n * D::NC + k);
        }
        if (do_aux) {
            double gn[D::NA * DIM];
            load_row<D::NA * DIM, double>(in.gab + (size_t)n * GR::AS, gn);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++)
#pragma unroll
                for (int d = 0; d < DIM; d++) ab[k] += wa[d] * gn[k * DIM + d];
        }
    }
    double u[D::NC];
    load_state<DIM, NS>(U, m, u);
    cell_aux_vjp<DIM, NS>(P, u, aux, m, ab, ub);
    bool finite = true;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        Ub[(size_t)m * D::NC + k] += ub[k];
        finite = finite && isfinite(ub[k]);
    }
    if (!finite) atomicOr(status, kStatusNaN);
}

}  // namespace abl
