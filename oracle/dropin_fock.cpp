// The engine dropped into the reference's own SCF classes: the binding a
// maintainer adds to aromanro/HartreeFock (the INTEGRATION guide's first
// section), compiled for real.  TEST INFRASTRUCTURE: oracle/Makefile (target
// dropin) links the reference's objects, compiled unmodified, with the member
// functions below weakened in copies of those objects (objcopy
// --weaken-symbol), so these definitions take their place:
//
//   IntegralsRepository::CalculateElectronElectronIntegrals
//       (IntegralsRepository.cpp:566-584): the packed 8-fold table from the
//       engine (hfg_eri_packed); with HFG_DROPIN_DIRECT no table at all;
//   RestrictedHartreeFock::InitFockMatrix (RestrictedHartreeFock.cpp:168-207)
//   UnrestrictedHartreeFock::InitFockMatrices (UnrestrictedHartreeFock.cpp:193-243)
//       with HFG_DROPIN_DIRECT only: G from the engine's direct build
//       (hfg_fock_rhf / hfg_fock_uhf); the iteration-0 guess as the reference
//       forms it.
//
// Everything else -- Basis, Molecule, the one-electron matrices, DIIS, the
// eigensolves, the convergence loop -- is the reference's own code.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <unordered_map>
#include <vector>

#include "IntegralsRepository.h"
#include "RestrictedHartreeFock.h"
#include "UnrestrictedHartreeFock.h"
#include "hfgpu.h"

namespace {

// one engine context per repository (the reference owns one repository per
// algorithm object, one algorithm per job thread)
thread_local std::unordered_map<const GaussianIntegrals::IntegralsRepository *, hfg_ctx *> g_ctx;

[[noreturn]] void die(const char *what) {
  std::fprintf(stderr, "%s: %s\n", what, hfg_last_error());
  std::exit(3);
}

hfg_ctx *context_for(const GaussianIntegrals::IntegralsRepository *repo, const Systems::Molecule *molecule) {
  auto it = g_ctx.find(repo);
  if (it != g_ctx.end()) {
    hfg_ctx_destroy(it->second);
    g_ctx.erase(it);
  }
  // IntegralsRepository::Reset(Molecule*) (IntegralsRepository.cpp:19-27):
  // the shell table, one engine shell per basis-file letter (an SP line is
  // two shells, L=0 and L=1, sharing exponents), in the reference's AO order
  std::vector<double> center, expo, coef;
  std::vector<int32_t> L, nprim, poff, aoff;
  int32_t ao = 0;
  for (const auto &atom : molecule->atoms)
    for (const auto &shell : atom.shells)
      for (size_t f = 0; f < shell.basisFunctions.size();) {
        const auto &cgo = shell.basisFunctions[f];  // first Cartesian component of this letter
        const int l = (int)cgo.angularMomentum.AngularMomentum();
        L.push_back(l);
        nprim.push_back((int32_t)cgo.gaussianOrbitals.size());
        poff.push_back((int32_t)expo.size());
        aoff.push_back(ao);
        center.insert(center.end(), {atom.position.X, atom.position.Y, atom.position.Z});
        for (const auto &g : cgo.gaussianOrbitals) {
          expo.push_back(g.alpha);
          coef.push_back(g.coefficient);
        }
        const int nc = (l + 1) * (l + 2) / 2;
        ao += nc;
        f += nc;
      }
  hfg_shells sh{(int32_t)L.size(), center.data(), L.data(), nprim.data(), poff.data(), aoff.data(),
                expo.data(), coef.data(), ao};
  hfg_opts o;
  hfg_default_opts(&o);  // Schwarz 1e-12, the reference's (dd|dd) convention
  hfg_ctx *ctx = nullptr;
  if (hfg_ctx_create(&sh, &o, &ctx) != HFG_OK) die("hfg_ctx_create");
  g_ctx[repo] = ctx;
  return ctx;
}

hfg_ctx *context_of(const GaussianIntegrals::IntegralsRepository *repo) {
  auto it = g_ctx.find(repo);
  if (it == g_ctx.end()) die("no engine context for this repository");
  return it->second;
}

// Eigen (column-major) <-> the engine's row-major n x n: symmetric matrices
// are the same array either way; copied element-wise for the shim's storage.
std::vector<double> row_major(const Eigen::MatrixXd &m) {
  std::vector<double> out((size_t)m.rows() * m.cols());
  for (long i = 0; i < m.rows(); ++i)
    for (long j = 0; j < m.cols(); ++j) out[(size_t)i * m.cols() + j] = m(i, j);
  return out;
}

void add_row_major(Eigen::MatrixXd &m, const std::vector<double> &a) {
  for (long i = 0; i < m.rows(); ++i)
    for (long j = 0; j < m.cols(); ++j) m(i, j) += a[(size_t)i * m.cols() + j];
}

}  // namespace

void GaussianIntegrals::IntegralsRepository::CalculateElectronElectronIntegrals() {
  hfg_ctx *ctx = context_for(this, m_Molecule);
#ifdef HFG_DROPIN_DIRECT
  (void)ctx;  // direct Fock builds: no table
#else
  const int n = (int)m_Molecule->CountNumberOfContractedGaussians();
  // the reference sizes the table GetElectronElectronIndex(N, N, N, N) + 1
  // (IntegralsRepository.cpp:568-571); the engine fills indices up to N - 1
  electronElectronIntegrals.resize((size_t)GetElectronElectronIndex(n, n, n, n) + 1);
  electronElectronIntegrals = 0.0;
  if (hfg_eri_packed(ctx, &electronElectronIntegrals[0], hfg_packed_size(n)) != HFG_OK) die("hfg_eri_packed");
#endif
}

#ifdef HFG_DROPIN_DIRECT
void HartreeFock::RestrictedHartreeFock::InitFockMatrix(int iter, Eigen::MatrixXd &FockMatrix) const {
  if (0 == iter) {
    if (initGuess > 0) {
      FockMatrix.resize(h.rows(), h.cols());
      for (int i = 0; i < h.rows(); ++i)
        for (int j = 0; j < h.rows(); ++j)
          FockMatrix(i, j) = initGuess * overlapMatrix.matrix(i, j) * (h(i, i) + h(j, j)) * 0.5;
    } else {
      FockMatrix = h;
    }
  } else {
    std::vector<double> G((size_t)h.rows() * h.cols());
    if (hfg_fock_rhf(context_of(&integralsRepository), row_major(DensityMatrix).data(), G.data()) != HFG_OK)
      die("hfg_fock_rhf");
    FockMatrix = h;
    add_row_major(FockMatrix, G);
  }
  FockMatrix = (FockMatrix + FockMatrix.transpose()) * 0.5;
}

void HartreeFock::UnrestrictedHartreeFock::InitFockMatrices(int iter, Eigen::MatrixXd &FockMatrixPlus,
                                                           Eigen::MatrixXd &FockMatrixMinus) const {
  if (0 == iter) {
    if (initGuess > 0) {
      FockMatrixPlus.resize(h.rows(), h.cols());
      FockMatrixMinus.resize(h.rows(), h.cols());
      for (int i = 0; i < h.rows(); ++i)
        for (int j = 0; j < h.rows(); ++j)
          FockMatrixPlus(i, j) = FockMatrixMinus(i, j) = initGuess * overlapMatrix.matrix(i, j) * (h(i, i) + h(j, j)) * 0.5;
    } else {
      FockMatrixPlus = h;
      FockMatrixMinus = h;
    }
    if (addAsymmetry && FockMatrixPlus.cols() > 1) {
      FockMatrixPlus(0, 1) += asymmetry;
      FockMatrixPlus(1, 0) = FockMatrixPlus(0, 1);
    }
  } else {
    std::vector<double> Gp((size_t)h.rows() * h.cols()), Gm(Gp.size());
    if (hfg_fock_uhf(context_of(&integralsRepository), row_major(DensityMatrixPlus).data(),
                     row_major(DensityMatrixMinus).data(), Gp.data(), Gm.data()) != HFG_OK)
      die("hfg_fock_uhf");
    FockMatrixPlus = h;
    FockMatrixMinus = h;
    add_row_major(FockMatrixPlus, Gp);
    add_row_major(FockMatrixMinus, Gm);
  }
}
#endif
