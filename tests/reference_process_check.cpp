// TEST INFRASTRUCTURE ONLY: drives the B200Rhs process (ablate_b200/reference_process) compiled against
// the reference-interface stand-ins of tests/reference_shim, linked with the product library.
// Built and run by tests/test_reference_process.py.
//
//   reference_process_check map
//       maps several configurations of the reference's objects (EOS, flux calculator, transport, the
//       PetscFV options) and prints one line per descriptor field; checks that Setup registers exactly
//       ComputeRhs with the process as its context ("registered 1").
//   reference_process_check rhs <mesh file> <state file> <out file> <flux> <limiter> <k> <mu>
//       builds a perfect-gas (1.4, 287) process with that flux calculator (ausm | ausmpup, mInf 0.3),
//       limiter (least squares) and constant transport, runs Setup and Initialize on the stand-in solver
//       holding the mesh, calls the solver's ComputeRHSFunction (which calls the registered function on
//       locX / locF) and writes F. Mesh file layout as tests/setup_records_check.cpp; state and F are
//       [n_cells][2 + dim] doubles. Exit code 3 with the PETSc error text when the call fails.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200Rhs.hpp"
#include "eos/perfectGas.hpp"
#include "eos/tChem.hpp"
#include "eos/transport/constant.hpp"
#include "eos/transport/sutherland.hpp"
#include "finiteVolume/fluxCalculator/ausm.hpp"
#include "finiteVolume/fluxCalculator/ausmpUp.hpp"
#include "finiteVolume/fluxCalculator/averageFlux.hpp"
#include "finiteVolume/fluxCalculator/offFlux.hpp"
#include "finiteVolume/fluxCalculator/riemann.hpp"

using namespace ablate;
using finiteVolume::processes::B200Rhs;

// the stand-in solver's mesh, copied into the process's LocalMesh
B200Rhs::LocalMesh finiteVolume::processes::GetLocalMesh(const finiteVolume::FiniteVolumeSolver& flow) {
    const abl_mesh_desc& m = flow.mesh;
    B200Rhs::LocalMesh lm;
    lm.dim = m.dim;
    lm.nCells = m.n_cells;
    lm.nFaces = m.n_faces;
    lm.faceCells.assign(m.face_cells, m.face_cells + 2 * (size_t)m.n_faces);
    lm.faceNormal.assign(m.face_normal, m.face_normal + 3 * (size_t)m.n_faces);
    lm.faceCentroid.assign(m.face_centroid, m.face_centroid + 3 * (size_t)m.n_faces);
    lm.cellCentroid.assign(m.cell_centroid, m.cell_centroid + 3 * (size_t)m.n_cells);
    lm.cellVolume.assign(m.cell_volume, m.cell_volume + (size_t)m.n_cells);
    if (m.cell_kind) lm.cellKind.assign(m.cell_kind, m.cell_kind + (size_t)m.n_cells);
    if (m.face_shift) lm.faceShift.assign(m.face_shift, m.face_shift + 3 * (size_t)m.n_faces);
    return lm;
}

static void print_physics(const char* name, const abl_physics_desc& p) {
    std::printf("%s eos=%d gamma=%.17g r_gas=%.17g n_species=%d flux=%d minf=%.17g pgs_alpha=%.17g recon=%d limiter=%d max_lim_grad=%.17g "
                "transport=%d k=%.17g mu=%.17g diff=%.17g advection=%d diffusion=%d species_advection=%d species_diffusion=%d compact=%d "
                "species_diff=%s nasa7=%s mw0=%.17g\n",
                name, p.eos, p.gamma, p.r_gas, p.n_species, p.flux, p.ausmpup_minf, p.pgs_alpha, p.reconstruction, p.limiter, p.max_lim_grad,
                p.transport, p.k, p.mu, p.diff, p.advection, p.diffusion, p.species_advection, p.species_diffusion, p.species_advection_compact,
                p.species_diff ? "set" : "null", p.nasa7 ? "set" : "null", p.mw ? p.mw[0] : 0.0);
}

static int map_mode() {
    {
        B200Rhs::Options o;
        o.limiter = "minmod";
        o.mInf = 0.3;
        B200Rhs p(std::make_shared<eos::PerfectGas>(1.4, 287.0), std::make_shared<finiteVolume::fluxCalculator::AusmpUp>(),
                  std::make_shared<eos::transport::Constant>(0.0252, 1.8e-5, 0.0), o);
        print_physics("ns_ausmpup_constant", p.Physics());
        finiteVolume::FiniteVolumeSolver flow;
        p.Setup(flow);
        const bool reg = flow.rhsArbitraryFunctions.size() == 1 && flow.rhsArbitraryFunctions[0].first == &B200Rhs::ComputeRhs &&
                         flow.rhsArbitraryFunctions[0].second == &p;
        std::printf("registered %d\n", reg ? 1 : 0);
    }
    {
        B200Rhs::Options o;
        o.reconstruction = "upwind";
        o.diffusion = false;
        B200Rhs p(std::make_shared<eos::PerfectGas>(1.3, 300.0, std::vector<std::string>{"A", "B"}), std::make_shared<finiteVolume::fluxCalculator::Ausm>(),
                  nullptr, o);
        print_physics("species_ausm_upwind", p.Physics());
    }
    {
        B200Rhs::Options o;
        o.limiter = "vanleer";
        o.compactSpeciesAdvection = true;
        o.nasa7.assign(15 * 3, 1.0);
        B200Rhs p(std::make_shared<eos::TChem>(std::vector<std::string>{"O2", "N2", "H2O"}, std::vector<double>{31.998, 28.014, 18.015}),
                  std::make_shared<finiteVolume::fluxCalculator::AverageFlux>(),
                  std::make_shared<eos::transport::Constant>(0.03, 2e-5, std::vector<double>{1e-5, 2e-5, 3e-5}), o);
        print_physics("tchem_average_vector_diff", p.Physics());
    }
    {
        B200Rhs::Options o;
        o.limiter = "sin";
        B200Rhs p(std::make_shared<eos::PerfectGas>(1.4, 287.0), std::make_shared<finiteVolume::fluxCalculator::Riemann>(),
                  std::make_shared<eos::transport::Sutherland>(), o);
        print_physics("riemann_sutherland", p.Physics());
    }
    {
        B200Rhs p(std::make_shared<eos::PerfectGas>(1.4, 287.0), std::make_shared<finiteVolume::fluxCalculator::OffFlux>(), nullptr, {});
        print_physics("off", p.Physics());
    }
    // configurations with no device counterpart are rejected at construction
    int rejected = 0;
    try {
        B200Rhs::Options o;
        o.limiter = "superbee";
        B200Rhs p(std::make_shared<eos::PerfectGas>(1.4, 287.0), nullptr, nullptr, o);
    } catch (const std::invalid_argument&) {
        rejected++;
    }
    try {
        B200Rhs p(std::make_shared<eos::TChem>(std::vector<std::string>{"O2"}, std::vector<double>{32.0}), nullptr, nullptr, {});
    } catch (const std::invalid_argument&) {
        rejected++;  // TChem without NASA-7 tables
    }
    std::printf("rejected %d\n", rejected);
    return 0;
}

template <class T>
static bool read_array(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

static int rhs_mode(int argc, char** argv) {
    if (argc != 9) return 2;
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) return 2;
    int32_t hdr[6];
    if (std::fread(hdr, sizeof(int32_t), 6, f) != 6) return 2;
    const int dim = hdr[0], nc = hdr[1], nf = hdr[2];
    const bool has_shift = hdr[3] != 0;
    std::vector<int32_t> fc;
    std::vector<double> fn, fcen, cc, cvol, fs;
    std::vector<uint8_t> ck;
    bool ok = read_array(f, fc, 2 * (size_t)nf) && read_array(f, fn, 3 * (size_t)nf) && read_array(f, fcen, 3 * (size_t)nf) &&
              read_array(f, cc, 3 * (size_t)nc) && read_array(f, cvol, (size_t)nc) && read_array(f, ck, (size_t)nc) &&
              (!has_shift || read_array(f, fs, 3 * (size_t)nf));
    std::fclose(f);
    const size_t nvals = (size_t)nc * (2 + dim);
    std::vector<double> X, F(nvals, 0.0);
    FILE* g = std::fopen(argv[3], "rb");
    ok = ok && g && read_array(g, X, nvals);
    if (g) std::fclose(g);
    if (!ok) return 2;

    B200Rhs::Options o;
    o.limiter = argv[6];
    o.mInf = 0.3;
    std::shared_ptr<finiteVolume::fluxCalculator::FluxCalculator> flux;
    if (std::strcmp(argv[5], "ausmpup") == 0)
        flux = std::make_shared<finiteVolume::fluxCalculator::AusmpUp>();
    else
        flux = std::make_shared<finiteVolume::fluxCalculator::Ausm>();
    B200Rhs process(std::make_shared<eos::PerfectGas>(1.4, 287.0), flux, std::make_shared<eos::transport::Constant>(std::atof(argv[7]), std::atof(argv[8]), 0.0), o);
    finiteVolume::FiniteVolumeSolver flow;
    flow.mesh = abl_mesh_desc{dim, nc, nf, fc.data(), fn.data(), fcen.data(), cc.data(), cvol.data(), ck.data(), has_shift ? fs.data() : nullptr};
    process.Setup(flow);
    try {
        process.Initialize(flow);
    } catch (const std::exception& e) {
        std::printf("initialize failed: %s\n", e.what());
        return 3;
    }
    _p_Vec locX{X.data(), (PetscInt)nvals}, locF{F.data(), (PetscInt)nvals};
    const PetscErrorCode e = flow.ComputeRHSFunction(0.0, &locX, &locF);
    if (e != PETSC_SUCCESS) {
        std::printf("rhs failed %d: %s\n", e, petsc_shim::last_error().c_str());
        return 3;
    }
    FILE* o_ = std::fopen(argv[4], "wb");
    if (!o_ || std::fwrite(F.data(), sizeof(double), nvals, o_) != nvals) return 2;
    std::fclose(o_);
    std::printf("rhs ok\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 2 && std::strcmp(argv[1], "map") == 0) return map_mode();
    if (argc >= 2 && std::strcmp(argv[1], "rhs") == 0) return rhs_mode(argc, argv);
    return 2;
}
