// Host side of the reference's C++ surface (include/hfgpu_host.hpp):
// basis files, molecules, one-electron integrals, the SCF driver and DIIS.
// Two-electron work goes to the GPU engine through the C ABI (hfgpu.h);
// the symmetric eigen-decompositions go to cuSOLVER.
#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <array>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "../../include/hfgpu_driver.h"
#include "../../include/hfgpu_host.hpp"
#include "driver_internal.h"
#include "scf_device.h"

namespace {

const char *kElements[] = {"H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg",
                           "Al", "Si", "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr",
                           "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr"};

unsigned z_for(const std::string &sym) {
  for (unsigned i = 0; i < sizeof kElements / sizeof kElements[0]; ++i)
    if (sym == kElements[i]) return i + 1;
  return 0;
}

int letter_l(char c) {
  switch (std::tolower(static_cast<unsigned char>(c))) {
    case 's': return 0;
    case 'p': return 1;
    case 'd': return 2;
    case 'f': return 3;
    case 'g': return 4;
    default: return -1;
  }
}

inline int ncart(int L) { return (L + 1) * (L + 2) / 2; }

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

}  // namespace

// ===========================================================================
// matrices and the GPU eigensolver
// ===========================================================================
namespace hfgpu {

namespace {
// cuBLAS handle and device buffers for the SCF's large matrix products
struct Gemm {
  cublasHandle_t h = nullptr;
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  size_t capA = 0, capB = 0, capC = 0;
  void release() {
    if (h) cublasDestroy(h);
    if (dA) cudaFree(dA);
    if (dB) cudaFree(dB);
    if (dC) cudaFree(dC);
    h = nullptr;
    dA = dB = dC = nullptr;
    capA = capB = capC = 0;
  }
  ~Gemm() { release(); }
};
Gemm &gemm_state() {
  static thread_local Gemm g;
  return g;
}
void grow(double **p, size_t *cap, size_t need) {
  if (need <= *cap) return;
  cudaFree(*p);
  *p = nullptr;
  if (cudaMalloc(p, need * sizeof(double)) != cudaSuccess) throw std::runtime_error("cudaMalloc (gemm)");
  *cap = need;
}
}  // namespace

Matrix operator*(const Matrix &a, const Matrix &b) {
  Matrix m(a.rows(), b.cols());
  const int n = a.rows(), p = a.cols(), q = b.cols();
  if ((double)n * p * q > 2.0e6) {
    // FP64 DGEMM on the GPU; row-major C = A B is column-major C^T = B^T A^T
    Gemm &g = gemm_state();
    if (!g.h && cublasCreate(&g.h) != CUBLAS_STATUS_SUCCESS) throw std::runtime_error("cublasCreate");
    grow(&g.dA, &g.capA, (size_t)n * p);
    grow(&g.dB, &g.capB, (size_t)p * q);
    grow(&g.dC, &g.capC, (size_t)n * q);
    if (cudaMemcpy(g.dA, a.data(), sizeof(double) * n * p, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g.dB, b.data(), sizeof(double) * p * q, cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy (gemm)");
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(g.h, CUBLAS_OP_N, CUBLAS_OP_N, q, n, p, &one, g.dB, q, g.dA, p, &zero, g.dC, q) !=
        CUBLAS_STATUS_SUCCESS)
      throw std::runtime_error("cublasDgemm");
    if (cudaMemcpy(m.data(), g.dC, sizeof(double) * n * q, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy (gemm)");
    return m;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < p; ++k) {
      const double aik = a(i, k);
      if (aik == 0.0) continue;
      const double *br = b.data() + (size_t)k * q;
      double *mr = m.data() + (size_t)i * q;
      for (int j = 0; j < q; ++j) mr[j] += aik * br[j];
    }
  return m;
}
Matrix operator+(const Matrix &a, const Matrix &b) {
  Matrix m = a;
  for (size_t x = 0; x < (size_t)a.rows() * a.cols(); ++x) m.data()[x] += b.data()[x];
  return m;
}
Matrix operator-(const Matrix &a, const Matrix &b) {
  Matrix m = a;
  for (size_t x = 0; x < (size_t)a.rows() * a.cols(); ++x) m.data()[x] -= b.data()[x];
  return m;
}
Matrix operator*(double s, const Matrix &a) {
  Matrix m = a;
  for (size_t x = 0; x < (size_t)a.rows() * a.cols(); ++x) m.data()[x] *= s;
  return m;
}
Matrix transpose(const Matrix &a) {
  Matrix t(a.cols(), a.rows());
  for (int i = 0; i < a.rows(); ++i)
    for (int j = 0; j < a.cols(); ++j) t(j, i) = a(i, j);
  return t;
}

namespace {
struct Solver {
  cusolverDnHandle_t h = nullptr;
  double *dA = nullptr, *dW = nullptr, *work = nullptr;
  int *info = nullptr;
  int cap = 0, lwork = 0;
  std::mutex mu;
  void release() {
    if (h) cusolverDnDestroy(h);
    if (dA) cudaFree(dA);
    if (dW) cudaFree(dW);
    if (work) cudaFree(work);
    if (info) cudaFree(info);
    h = nullptr;
    dA = dW = work = nullptr;
    info = nullptr;
    cap = lwork = 0;
  }
  ~Solver() { release(); }
};
Solver &solver() {
  static thread_local Solver s;
  return s;
}
void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void check_solver(cusolverStatus_t e, const char *what) {
  if (e != CUSOLVER_STATUS_SUCCESS) throw std::runtime_error(std::string(what) + " failed");
}
}  // namespace

// Frees this host thread's library handles and buffers while the thread (and
// CUDA) are alive: a thread that exits otherwise frees them in its
// thread-local destructors, which can run after the process has begun to
// tear CUDA down.
void release_thread_state() {
  gemm_state().release();
  solver().release();
}

void eigh(const Matrix &a, std::vector<double> &w, Matrix &v) {
  const int n = a.rows();
  Solver &s = solver();
  if (!s.h) check_solver(cusolverDnCreate(&s.h), "cusolverDnCreate");
  if (n > s.cap) {
    cudaFree(s.dA);
    cudaFree(s.dW);
    cudaFree(s.work);
    cudaFree(s.info);
    check_cuda(cudaMalloc(&s.dA, sizeof(double) * n * n), "cudaMalloc");
    check_cuda(cudaMalloc(&s.dW, sizeof(double) * n), "cudaMalloc");
    check_cuda(cudaMalloc(&s.info, sizeof(int)), "cudaMalloc");
    check_solver(cusolverDnDsyevd_bufferSize(s.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, s.dA, n, s.dW,
                                             &s.lwork),
                 "dsyevd_bufferSize");
    check_cuda(cudaMalloc(&s.work, sizeof(double) * s.lwork), "cudaMalloc");
    s.cap = n;
  }
  // symmetric input: row-major == column-major
  check_cuda(cudaMemcpy(s.dA, a.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice), "cudaMemcpy");
  check_solver(cusolverDnDsyevd(s.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, s.dA, n, s.dW, s.work,
                                s.lwork, s.info),
               "dsyevd");
  std::vector<double> colmajor((size_t)n * n);
  w.resize(n);
  int info = 0;
  check_cuda(cudaMemcpy(colmajor.data(), s.dA, sizeof(double) * n * n, cudaMemcpyDeviceToHost), "cudaMemcpy");
  check_cuda(cudaMemcpy(w.data(), s.dW, sizeof(double) * n, cudaMemcpyDeviceToHost), "cudaMemcpy");
  check_cuda(cudaMemcpy(&info, s.info, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
  if (info != 0) throw std::runtime_error("dsyevd did not converge");
  v.resize(n, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) v(i, j) = colmajor[(size_t)j * n + i];
}

}  // namespace hfgpu

// ===========================================================================
// basis, atoms, molecule
// ===========================================================================
unsigned Orbitals::ContractedGaussianShell::CountNumberOfContractedGaussians() const {
  unsigned n = 0;
  for (char c : letters) n += ncart(letter_l(c));
  return n;
}

unsigned Systems::AtomWithShells::CountNumberOfContractedGaussians() const {
  unsigned n = 0;
  for (const auto &s : shells) n += s.CountNumberOfContractedGaussians();
  return n;
}

unsigned Systems::AtomWithShells::GetMaxAngularMomentum() const {
  int L = 0;
  for (const auto &s : shells)
    for (char c : s.letters) L = std::max(L, letter_l(c));
  return (unsigned)L;
}

void Chemistry::Basis::Load(const std::string &fileName) {
  std::ifstream f(fileName);
  if (!f) throw std::runtime_error("cannot open basis file " + fileName);
  atoms.clear();
  std::string line;
  Orbitals::ContractedGaussianShell *cur = nullptr;
  while (std::getline(f, line)) {
    const std::string t = trim(line);
    if (t.empty() || t[0] == '#' || t.rfind("BASIS", 0) == 0 || t.rfind("END", 0) == 0) continue;
    std::istringstream ls(t);
    std::string a, b, extra;
    ls >> a >> b;
    const bool shell_line = std::isalpha(static_cast<unsigned char>(a[0])) && !b.empty() &&
                            std::isalpha(static_cast<unsigned char>(b[0])) && !(ls >> extra);
    if (shell_line) {
      const unsigned Z = z_for(a);
      if (!Z) throw std::runtime_error("unknown element " + a + " in " + fileName);
      if (atoms.empty() || atoms.back().Z != Z) atoms.emplace_back(Z);
      for (char c : b)
        if (letter_l(c) < 0) throw std::runtime_error("unknown shell letter in " + fileName);
      atoms.back().shells.push_back(Orbitals::ContractedGaussianShell{b, {}, std::vector<std::vector<double>>(b.size())});
      cur = &atoms.back().shells.back();
      continue;
    }
    if (!cur) continue;
    std::string num;
    std::istringstream ns(t);
    std::vector<double> vals;
    while (ns >> num) {
      std::replace(num.begin(), num.end(), 'D', 'E');
      vals.push_back(std::stod(num));
    }
    if (vals.empty()) continue;
    cur->exponents.push_back(vals[0]);
    for (size_t i = 0; i < cur->letters.size() && i + 1 < vals.size(); ++i) cur->coefficients[i].push_back(vals[i + 1]);
  }
}

unsigned Systems::Molecule::CountNumberOfContractedGaussians() const {
  unsigned n = 0;
  for (const auto &a : atoms) n += a.CountNumberOfContractedGaussians();
  return n;
}

unsigned Systems::Molecule::ElectronsNumber() const {
  if (alphaElectrons > 0 || betaElectrons > 0) return alphaElectrons + betaElectrons;
  unsigned n = 0;
  for (const auto &a : atoms) n += a.electronsNumber;
  return n;
}

unsigned Systems::Molecule::GetMaxAngularMomentum() const {
  unsigned L = 0;
  for (const auto &a : atoms) L = std::max(L, a.GetMaxAngularMomentum());
  return L;
}

double Systems::Molecule::NuclearRepulsionEnergy() const {
  double e = 0;
  for (size_t i = 0; i < atoms.size(); ++i)
    for (size_t j = i + 1; j < atoms.size(); ++j) {
      const double dx = atoms[i].position.X - atoms[j].position.X, dy = atoms[i].position.Y - atoms[j].position.Y,
                   dz = atoms[i].position.Z - atoms[j].position.Z;
      e += double(atoms[i].Z) * atoms[j].Z / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  return e;
}

double Systems::Molecule::NuclearElectricFieldEnergy() const {
  double e = 0;
  for (const auto &a : atoms)
    e -= double(a.Z) * (a.position.X * ElectricField.X + a.position.Y * ElectricField.Y + a.position.Z * ElectricField.Z);
  return e;
}

void Systems::Molecule::Init() {
  ShellTable t;
  int ao = 0;
  for (size_t a = 0; a < atoms.size(); ++a) {
    atoms[a].ID = (unsigned)a;
    for (const auto &sh : atoms[a].shells)
      for (size_t li = 0; li < sh.letters.size(); ++li) {
        const int L = letter_l(sh.letters[li]);
        t.center.push_back(atoms[a].position.X);
        t.center.push_back(atoms[a].position.Y);
        t.center.push_back(atoms[a].position.Z);
        t.L.push_back(L);
        t.nprim.push_back((int32_t)sh.exponents.size());
        t.prim_offset.push_back((int32_t)t.exponent.size());
        t.ao_offset.push_back(ao);
        t.exponent.insert(t.exponent.end(), sh.exponents.begin(), sh.exponents.end());
        t.coefficient.insert(t.coefficient.end(), sh.coefficients[li].begin(), sh.coefficients[li].end());
        ao += ncart(L);
      }
  }
  t.nbf = ao;
  table_ = std::move(t);
  // occupations, Molecule.cpp:132-139
  const unsigned el = ElectronsNumber();
  if (alphaElectrons == 0 && betaElectrons == 0) {
    alphaElectrons = el / 2;
    betaElectrons = el - alphaElectrons;
  }
}

hfg_shells Systems::Molecule::ShellTable::view() const {
  hfg_shells s{};
  s.nshells = (int32_t)L.size();
  s.center = center.data();
  s.L = L.data();
  s.nprim = nprim.data();
  s.prim_offset = prim_offset.data();
  s.ao_offset = ao_offset.data();
  s.exponent = exponent.data();
  s.coefficient = coefficient.data();
  s.nbf = nbf;
  return s;
}

// Molecule::LoadXYZ (Molecule.cpp:143-199): count line, comment line, then
// "symbol x y z" per atom with the coordinates as written; false on a short
// file, an unknown symbol, an element the basis lacks, or a count line that
// does not parse (the reference's catch-all).
bool Systems::Molecule::LoadXYZ(const std::string &fileName, const Chemistry::Basis &basis) {
  try {
    return LoadXYZBody(fileName, basis);
  } catch (...) {
  }
  return false;
}

bool Systems::Molecule::LoadXYZBody(const std::string &fileName, const Chemistry::Basis &basis) {
  std::ifstream f(fileName);
  if (!f) return false;
  std::string line;
  if (!std::getline(f, line)) return false;
  const unsigned n = (unsigned)std::stoi(line);
  if (!std::getline(f, line)) return false;
  for (unsigned i = 0; i < n; ++i) {
    if (!std::getline(f, line)) return false;
    std::istringstream ls(line);
    std::string sym;
    double x, y, z;
    ls >> sym >> x >> y >> z;
    const unsigned Z = z_for(sym);
    bool found = false;
    for (const auto &a : basis.atoms)
      if (a.Z == Z) {
        atoms.push_back(a);
        atoms.back().position = {x, y, z};
        found = true;
        break;
      }
    if (!found) return false;
  }
  Init();
  return true;
}

// ===========================================================================
// IntegralsRepository
// ===========================================================================
namespace GaussianIntegrals {

IntegralsRepository::IntegralsRepository(Systems::Molecule *molecule) : molecule_(molecule) {
  hfg_default_opts(&options);
}

IntegralsRepository::~IntegralsRepository() {
  if (ctx_) hfg_ctx_destroy(ctx_);
}

void IntegralsRepository::Reset(Systems::Molecule *molecule) {
  if (ctx_) hfg_ctx_destroy(ctx_);
  ctx_ = nullptr;
  packed_.clear();
  packed_.shrink_to_fit();
  molecule_ = molecule;
}

hfg_ctx *IntegralsRepository::engine() {
  if (!ctx_) {
    if (!molecule_) throw std::runtime_error("IntegralsRepository without a molecule");
    const hfg_shells sh = molecule_->shellTable().view();
    if (hfg_ctx_create(&sh, &options, &ctx_) != HFG_OK)
      throw std::runtime_error(std::string("hfg_ctx_create: ") + hfg_last_error());
  }
  return ctx_;
}

void IntegralsRepository::CalculateElectronElectronIntegrals() {
  const int n = (int)molecule_->shellTable().nbf;
  packed_.assign((size_t)hfg_packed_size(n), 0.0);
  if (hfg_eri_packed(engine(), packed_.data(), (int64_t)packed_.size()) != HFG_OK)
    throw std::runtime_error(std::string("hfg_eri_packed: ") + hfg_last_error());
}

double IntegralsRepository::getElectronElectron(int i, int j, int k, int l) const {
  auto tri = [](long long a, long long b) { return a < b ? b * (b + 1) / 2 + a : a * (a + 1) / 2 + b; };
  return packed_[(size_t)tri(tri(i, j), tri(k, l))];
}

double IntegralsRepository::getElectronElectronDirect(int i, int j, int k, int l) {
  double v = 0;
  if (hfg_eri_quartet(engine(), i, j, k, l, &v) != HFG_OK)
    throw std::runtime_error(std::string("hfg_eri_quartet: ") + hfg_last_error());
  return v;
}

// QuantumMatrix.cpp:34-155 (overlap, kinetic, nuclear attraction): all
// shell pairs on the device (hfg_one_electron)
void IntegralsRepository::OneElectron(hfgpu::Matrix &S, hfgpu::Matrix &T, hfgpu::Matrix &V) const {
  const auto &t = molecule_->shellTable();
  const int n = t.nbf;
  S.resize(n, n);
  T.resize(n, n);
  V.resize(n, n);
  std::vector<double> nxyz;
  std::vector<int32_t> nz;
  for (const auto &a : molecule_->atoms) {
    nxyz.insert(nxyz.end(), {a.position.X, a.position.Y, a.position.Z});
    nz.push_back((int32_t)a.Z);
  }
  const hfg_shells sh = t.view();
  if (hfg_one_electron(&sh, nxyz.data(), nz.data(), (int32_t)nz.size(), options.device, S.data(), T.data(),
                       V.data()) != HFG_OK)
    throw std::runtime_error(std::string("hfg_one_electron: ") + hfg_last_error());
}

double MolecularOrbitalsIntegralsRepository::getElectronElectron(unsigned p, unsigned q, unsigned r, unsigned s,
                                                                  const hfgpu::Matrix &C) {
  if (mo_.empty()) {
    hfg_ctx *ctx = repo_.engine();
    n_ = hfg_ctx_nbf(ctx);
    if (C.rows() != n_ || C.cols() != n_) throw std::invalid_argument("MO coefficients: nbf x nbf expected");
    const size_t nn = (size_t)n_ * n_;
    double *dC = nullptr, *dX = nullptr;
    if (cudaMalloc(&dC, nn * sizeof(double)) != cudaSuccess || cudaMalloc(&dX, nn * nn * sizeof(double)) != cudaSuccess) {
      cudaFree(dC);
      throw std::runtime_error("MolecularOrbitalsIntegralsRepository: device allocation");
    }
    cudaMemcpy(dC, C.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
    const hfg_status st = hfg_mo_eri_full(ctx, dC, dX, nullptr);
    mo_.resize(nn * nn);
    if (st == HFG_OK) cudaMemcpy(mo_.data(), dX, nn * nn * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dC);
    cudaFree(dX);
    if (st != HFG_OK) {
      mo_.clear();
      throw std::runtime_error(std::string("hfg_mo_eri_full: ") + hfg_last_error());
    }
  }
  const size_t n = (size_t)n_;
  return mo_[((size_t)p * n + q) * n * n + (size_t)r * n + s];
}

SpinOrbitalsElectronElectronIntegralsRepository::SpinOrbitalsElectronElectronIntegralsRepository(int numOrbitals)
    : m_(2 * (size_t)numOrbitals), t_(m_ * m_ * m_ * m_, 0.0) {}

SpinOrbitalsElectronElectronIntegralsRepository::SpinOrbitalsElectronElectronIntegralsRepository(
    int numOrbitals, IntegralsRepository &repository, const hfgpu::Matrix &C)
    : SpinOrbitalsElectronElectronIntegralsRepository(numOrbitals) {
  Compute(repository, C);
}

void SpinOrbitalsElectronElectronIntegralsRepository::Compute(IntegralsRepository &repository, const hfgpu::Matrix &C) {
  hfg_ctx *ctx = repository.engine();
  if ((size_t)2 * hfg_ctx_nbf(ctx) != m_) throw std::invalid_argument("spin-orbital tensor: 2 nbf spin orbitals expected");
  if (hfg_spin_orbital_eri(ctx, C.data(), t_.data(), (int64_t)t_.size()) != HFG_OK)
    throw std::runtime_error(std::string("hfg_spin_orbital_eri: ") + hfg_last_error());
}

void IntegralsRepository::Moments(hfgpu::Matrix &Mx, hfgpu::Matrix &My, hfgpu::Matrix &Mz) const {
  const auto &t = molecule_->shellTable();
  const int n = t.nbf;
  Mx.resize(n, n);
  My.resize(n, n);
  Mz.resize(n, n);
  const hfg_shells sh = t.view();
  if (hfg_moments(&sh, options.device, Mx.data(), My.data(), Mz.data()) != HFG_OK)
    throw std::runtime_error(std::string("hfg_moments: ") + hfg_last_error());
}

}  // namespace GaussianIntegrals

// ===========================================================================
// SCF
// ===========================================================================
namespace HartreeFock {

using hfgpu::Matrix;

namespace {
// throws std::runtime_error with the engine's message unless st is HFG_OK
void check_engine(hfg_status st, const char *what);
}  // namespace

// Constants.h:6-10
constexpr double kEnergyConvergenceDIIS = 1E-11;
constexpr double kEnergyConvergence = 1E-13;
constexpr double kRmsDConvergence = 1E-10;
constexpr double kDiisConvergence = 1E-10;

HartreeFockAlgorithm::HartreeFockAlgorithm(int iterations)
    : totalEnergy(std::numeric_limits<double>::infinity()), maxIterations(iterations) {}

HartreeFockAlgorithm::~HartreeFockAlgorithm() = default;

void HartreeFockAlgorithm::Init(Systems::Molecule *molecule) {
  const auto t_init = std::chrono::steady_clock::now();
  converged = false;
  if (PrecisionForm()) {
    integralsRepository.options.incremental = 1;
    integralsRepository.options.density_screening = 1;
    integralsRepository.options.mixed_cutoff = std::max(0.0, mixedCutoff);
  }
  // the SCF's builds reuse one density and one G buffer: with cudaGraphs they
  // replay as a graph (one host thread driving the device); concurrentClasses
  // spreads a build's classes over streams
  integralsRepository.options.cuda_graphs = cudaGraphs ? 1 : 0;
  integralsRepository.options.concurrent_classes = concurrentClasses ? 1 : 0;
  integralsRepository.Reset(molecule);
  Matrix T, Vn;
  integralsRepository.OneElectron(overlap, T, Vn);
  integralsRepository.Moments(momentX, momentY, momentZ);
  // h = T + V + E . moments (HartreeFockAlgorithm.cpp:38)
  h = T + Vn;
  const hfgpu::Vector3D &E = molecule->ElectricField;
  if (E.X != 0 || E.Y != 0 || E.Z != 0) h = h + E.X * momentX + E.Y * momentY + E.Z * momentZ;
  molecule_ = molecule;
  nuclearRepulsionEnergy = molecule->NuclearRepulsionEnergy();
  nuclearElectricFieldEnergy = molecule->NuclearElectricFieldEnergy();
  numberOfOrbitals = (int)molecule->shellTable().nbf;
  // the reference always stores the 8-fold table at Init
  // (HartreeFockAlgorithm.cpp:45); it is kept here when it fits the budget
  if ((size_t)hfg_packed_size(numberOfOrbitals) * sizeof(double) <= storedIntegralsBudget)
    integralsRepository.CalculateElectronElectronIntegrals();
  else
    integralsRepository.engine();
  if (shardCount > 1) {
    if (!allReduce) throw std::invalid_argument("sharded SCF without an all-reduce of G");
    check_engine(hfg_set_shard(integralsRepository.engine(), shardRank, shardCount), "hfg_set_shard");
  }
  // V = S^-1/2 = U s^-1/2 U^T, symmetrised (HartreeFockAlgorithm.cpp:48-59)
  std::vector<double> w;
  Matrix U;
  hfgpu::eigh(overlap, w, U);
  const int n = numberOfOrbitals;
  Matrix Us(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Us(i, j) = U(i, j) / std::sqrt(w[j]);
  V = Us * hfgpu::transpose(U);
  Vt = hfgpu::transpose(V);
  V = Vt = 0.5 * (V + Vt);
  inited = true;
  secondsInit = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_init).count();
}

hfgpu::Vector3D HartreeFockAlgorithm::GetNuclearMoment() const {
  hfgpu::Vector3D m;
  if (!molecule_) return m;
  for (const auto &a : molecule_->atoms) {
    m.X += double(a.Z) * a.position.X;
    m.Y += double(a.Z) * a.position.Y;
    m.Z += double(a.Z) * a.position.Z;
  }
  return m;
}

namespace {
hfgpu::Vector3D electronic_moment(hfgpu::Vector3D m, const Matrix &P, const Matrix *P2, const Matrix &Mx,
                                  const Matrix &My, const Matrix &Mz) {
  const int n = P.rows();
  if (Mx.rows() != n) return m;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double d = P(i, j) + (P2 ? (*P2)(i, j) : 0.0);
      m.X -= d * Mx(i, j);
      m.Y -= d * My(i, j);
      m.Z -= d * Mz(i, j);
    }
  return m;
}
}  // namespace

double HartreeFockAlgorithm::Calculate() {
  double curEnergy = 0, prevEnergy = std::numeric_limits<double>::infinity();
  if (!inited) return prevEnergy;
  const auto t0 = std::chrono::steady_clock::now();
  fockMilliseconds = 0;
  fockBuilds = mixedSteps = 0;
  fp32Quartets = fp64Quartets = 0;
  secondsFock = secondsEigen = secondsDiis = secondsTotal = 0;
  fp64Phase = !PrecisionCriteria();
  fp64Steps = 0;
  if (PrecisionForm()) {
    hfg_ctx *ctx = integralsRepository.engine();
    if (hfg_set_mixed_cutoff(ctx, std::max(0.0, mixedCutoff)) != HFG_OK || hfg_set_incremental(ctx, 1) != HFG_OK)
      throw std::runtime_error(std::string("precision form: ") + hfg_last_error());
  }
  struct TotalTimer {
    double &out;
    std::chrono::steady_clock::time_point t0;
    ~TotalTimer() { out = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
  } total_timer{secondsTotal, t0};
  // the iterations run on the device; the public fields are synced around them
  Device().reset_timers();
  SyncToDevice();
  struct CalcScope {
    HartreeFockAlgorithm *a;
    bool done = false;
    ~CalcScope() {
      a->inCalculate = false;
      a->secondsEigen = a->device_ ? a->device_->eigen_seconds() : 0.0;
      if (!done) {
        try {
          a->SyncFromDevice();
        } catch (...) {
        }
      }
    }
  } scope{this};
  inCalculate = true;
  int iter = 0;
  FirstIterations(iter, curEnergy, prevEnergy);
  if (terminate) return curEnergy;
  // the reference's post-DIIS plain iterations (HartreeFockAlgorithm.cpp:117-121);
  // the precision form ends with its FP64 iterations instead
  const bool postDiis = !PrecisionCriteria() || fp64FinalConverge;
  if (postDiis && UseDIIS && iter < maxDIISiterations && converged && normalIterAfterDIIS) {
    SelfConsistentIterations(iter, curEnergy, prevEnergy);
    if (terminate) return curEnergy;
  }
  NormalIterations(iter, curEnergy, prevEnergy);
  iterations = iter;
  SyncFromDevice();
  scope.done = true;
  return curEnergy;
}

// Plain form: the reference's test.  Precision form: leave the incremental
// phase on its own (looser) test; from then on every build is a full FP64
// build from the whole density, and the SCF is done after
// fp64FinalIterations of them (or, with fp64FinalConverge, once the
// reference's test passes as well).
bool HartreeFockAlgorithm::ConvergedAfterStep(bool test, double dE, double rmsD) {
  if (!PrecisionCriteria()) return test;
  if (fp64Phase) return fp64Steps >= fp64FinalIterations && (test || !fp64FinalConverge);
  // a small step alone is not enough: a stalled DIIS also takes small steps
  if (test || (dE < mixedSwitchEnergy && rmsD < mixedSwitchDensity && lastErrorEst < mixedSwitchDiis)) {
    if (PrecisionForm()) {
      hfg_ctx *ctx = integralsRepository.engine();
      if (hfg_set_mixed_cutoff(ctx, 0.0) != HFG_OK || hfg_set_incremental(ctx, 0) != HFG_OK)
        throw std::runtime_error(std::string("precision form: ") + hfg_last_error());
    }
    fp64Phase = true;
    fp64Steps = 0;
  }
  return false;
}

void HartreeFockAlgorithm::TraceStep(int iter, double energy, double dE, double rmsD) const {
  if (!traceIterations) return;
  std::fprintf(stderr, "scf iter %4d E %.12f dE %.3e rmsD %.3e diis %.3e phase %s build_ms %.3f\n", iter, energy, dE,
               rmsD, lastErrorEst, fp64Phase ? "fp64" : (mixedCutoff > 0 ? "mixed" : "inc64"),
               fockBuilds ? fockMilliseconds / fockBuilds : 0.0);
}

void HartreeFockAlgorithm::AccountFockBuild() {
  hfg_stats st{};
  if (hfg_ctx_stats(integralsRepository.engine(), &st) != HFG_OK)
    throw std::runtime_error(std::string("hfg_ctx_stats: ") + hfg_last_error());
  fockMilliseconds += st.last_build_ms;
  ++fockBuilds;
  fp32Quartets += st.fp32_shell_quartets;
  fp64Quartets += st.fp64_shell_quartets;
  if (fp64Phase) ++fp64Steps;
  else ++mixedSteps;
}

void HartreeFockAlgorithm::FirstIterations(int &iter, double &curEnergy, double &prevEnergy) {
  for (; iter < maxIterations; ++iter) {
    const double rmsD = Step(iter);
    curEnergy = GetTotalEnergy();
    const double dE = std::fabs(prevEnergy - curEnergy);
    TraceStep(iter, curEnergy, dE, rmsD);
    const bool test = dE <= (UseDIIS ? kEnergyConvergenceDIIS : kEnergyConvergence) && rmsD < kRmsDConvergence &&
                      lastErrorEst < kDiisConvergence;
    if (ConvergedAfterStep(test, dE, rmsD)) {
      converged = true;
      break;
    }
    if (terminate) return;
    prevEnergy = curEnergy;
  }
}

void HartreeFockAlgorithm::SelfConsistentIterations(int &iter, double &curEnergy, double &prevEnergy) {
  UseDIIS = false;
  for (int i = 0; i < normalIterAfterDIIS; ++i) {
    Step(iter + i);
    curEnergy = GetTotalEnergy();
    if (terminate) {
      UseDIIS = true;
      return;
    }
    prevEnergy = curEnergy;
  }
  iter += normalIterAfterDIIS;
  UseDIIS = true;
}

void HartreeFockAlgorithm::NormalIterations(int &iter, double &curEnergy, double &prevEnergy) {
  if (converged) return;
  for (; iter < maxIterations; ++iter) {
    const double rmsD = Step(iter);
    curEnergy = GetTotalEnergy();
    const double dE = std::fabs(prevEnergy - curEnergy);
    TraceStep(iter, curEnergy, dE, rmsD);
    const bool test = dE <= kEnergyConvergence && rmsD < kRmsDConvergence;
    if (ConvergedAfterStep(test, dE, rmsD)) {
      converged = true;
      return;
    }
    if (terminate) return;
    prevEnergy = curEnergy;
  }
}

// DIIS.h:9-96: keep 6, extrapolate from 5, Pulay B matrix solved by a
// column-pivoted Householder QR
bool Diis::AddValueAndError(const Matrix &value, const Matrix &error) {
  errors_.push_back(error);
  values_.push_back(value);
  if (errors_.size() > 6) {
    errors_.erase(errors_.begin());
    values_.erase(values_.begin());
  }
  return errors_.size() >= 5;
}

namespace {
double dot(const Matrix &a, const Matrix &b) {
  double s = 0;
  for (size_t x = 0; x < (size_t)a.rows() * a.cols(); ++x) s += a.data()[x] * b.data()[x];
  return s;
}
}  // namespace
}  // namespace HartreeFock

// least-squares solve of a small dense system by column-pivoted Householder QR
std::vector<double> hfgpu::detail::pulay_solve(std::vector<double> A, int m, std::vector<double> b) {
  const int n = m;
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  auto at = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
  std::vector<std::vector<double>> hv;
  std::vector<double> betas;
  std::vector<int> ks;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = -1;
    for (int j = k; j < n; ++j) {
      double s = 0;
      for (int i = k; i < m; ++i) s += at(i, j) * at(i, j);
      if (s > best) { best = s; p = j; }
    }
    if (p != k) {
      for (int i = 0; i < m; ++i) std::swap(at(i, k), at(i, p));
      std::swap(perm[k], perm[p]);
    }
    double al = 0;
    for (int i = k; i < m; ++i) al += at(i, k) * at(i, k);
    al = std::sqrt(al);
    if (al == 0) continue;
    if (at(k, k) > 0) al = -al;
    std::vector<double> v(m - k);
    v[0] = at(k, k) - al;
    for (int i = k + 1; i < m; ++i) v[i - k] = at(i, k);
    double vn = 0;
    for (double x : v) vn += x * x;
    const double beta = vn > 0 ? 2.0 / vn : 0.0;
    for (int j = k; j < n; ++j) {
      double s = 0;
      for (int i = k; i < m; ++i) s += v[i - k] * at(i, j);
      s *= beta;
      for (int i = k; i < m; ++i) at(i, j) -= s * v[i - k];
    }
    double s = 0;
    for (int i = k; i < m; ++i) s += v[i - k] * b[i];
    s *= beta;
    for (int i = k; i < m; ++i) b[i] -= s * v[i - k];
  }
  const double tol = std::fabs(at(0, 0)) * 1e-15 * n;
  int rank = 0;
  while (rank < n && std::fabs(at(rank, rank)) > tol) ++rank;
  std::vector<double> z(n, 0.0), x(n, 0.0);
  for (int i = rank - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < rank; ++j) s -= at(i, j) * z[j];
    z[i] = s / at(i, i);
  }
  for (int j = 0; j < n; ++j) x[perm[j]] = z[j];
  return x;
}

namespace HartreeFock {

double Diis::Estimate(Matrix &value) const {
  const int nm = (int)errors_.size(), np1 = nm + 1;
  std::vector<double> B((size_t)np1 * np1, 0.0), rhs(np1, 0.0);
  double last = 0;
  for (int i = 0; i < nm; ++i) {
    for (int j = 0; j < i; ++j) B[i * np1 + j] = B[j * np1 + i] = dot(errors_[i], errors_[j]);
    B[i * np1 + i] = dot(errors_[i], errors_[i]);
    if (i == nm - 1 || i == nm - 2) last += B[i * np1 + i];
    B[nm * np1 + i] = B[i * np1 + nm] = 1;
  }
  last = std::sqrt(last);
  rhs[nm] = 1;
  const std::vector<double> c = hfgpu::detail::pulay_solve(B, np1, rhs);
  value = Matrix::Zero(value.rows(), value.cols());
  for (int i = 0; i < nm; ++i) value = value + c[i] * values_[i];
  return last;
}

namespace {
struct ScopedSeconds {
  double &acc;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit ScopedSeconds(double &a) : acc(a) {}
  ~ScopedSeconds() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};
void check_engine(hfg_status st, const char *what) {
  if (st != HFG_OK) throw std::runtime_error(std::string(what) + ": " + hfg_last_error());
}
// iteration-0 Fock matrix (RestrictedHartreeFock.cpp:175-186): the extended
// Hueckel-like guess initGuess S_ij (h_ii + h_jj)/2, or h when initGuess = 0
Matrix guess_fock(const Matrix &h, const Matrix &S, double initGuess) {
  if (!(initGuess > 0)) return h;
  const int n = h.rows();
  Matrix F(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) F(i, j) = initGuess * S(i, j) * (h(i, i) + h(j, j)) * 0.5;
  return F;
}
double occupied_sum(const std::vector<double> &w, const std::vector<bool> &occupied) {
  double e = 0;
  for (size_t l = 0; l < occupied.size() && l < w.size(); ++l)
    if (occupied[l]) e += w[l];
  return e;
}
}  // namespace

hfgpu::detail::DeviceScf &HartreeFockAlgorithm::Device() {
  if (!device_) {
    device_.reset(new hfgpu::detail::DeviceScf(numberOfOrbitals, integralsRepository.options.device));
    device_->SetMatrices(h.data(), overlap.data(), V.data());
  }
  return *device_;
}

void HartreeFockAlgorithm::AccountDevice(double fock_wall_seconds) {
  secondsFock += fock_wall_seconds;
  AccountFockBuild();
}

void RestrictedHartreeFock::Init(Systems::Molecule *molecule) {
  HartreeFockAlgorithm::Init(molecule);
  DensityMatrix = Matrix::Zero(h.rows(), h.cols());
  diis = Diis();
  nrOccupiedLevels = molecule->ElectronsNumber() / 2;  // RestrictedHartreeFock.cpp:24-31
  if (!nrOccupiedLevels) nrOccupiedLevels = 1;
  if (nrOccupiedLevels > (unsigned)numberOfOrbitals) nrOccupiedLevels = numberOfOrbitals;
  occupied.assign(nrOccupiedLevels, true);
  device_.reset();
  Device().ResetDiis();
}

void RestrictedHartreeFock::SyncToDevice() { Device().SetDensity(0, DensityMatrix.data()); }

void RestrictedHartreeFock::SyncFromDevice() {
  const int n = numberOfOrbitals;
  DensityMatrix.resize(n, n);
  C.resize(n, n);
  Device().CopyOut(0, DensityMatrix.data(), C.data());
}

// RestrictedHartreeFock::Step (RestrictedHartreeFock.cpp:61-166) with the
// matrices on the device: F (guess, or h + G from the direct build, then
// symmetrised), DIIS, F' = V F V, eigen-decomposition, C = V C', the new
// density 2 C_occ C_occ^T, the energy, the density change and the mixing.
double RestrictedHartreeFock::Step(int iter) {
  hfgpu::detail::DeviceScf &d = Device();
  if (!inCalculate) SyncToDevice();
  const int n = numberOfOrbitals;
  if (iter == 0) {
    Matrix F = guess_fock(h, overlap, initGuess);
    F = 0.5 * (F + hfgpu::transpose(F));
    d.SetFock(0, F.data());
  } else {
    const auto t0 = std::chrono::steady_clock::now();
    check_engine(hfg_fock_rhf_device(integralsRepository.engine(), d.density(0), d.g_buffer(0), d.stream()),
                 "hfg_fock_rhf_device");
    if (shardCount > 1) allReduce(d.g_buffer(0), (size_t)numberOfOrbitals * numberOfOrbitals, d.stream());
    AccountDevice(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    d.FockFromG(0, d.g_buffer(0), true);
  }
  bool used = false;
  if (UseDIIS && iter && iter < maxDIISiterations) {  // RestrictedHartreeFock.cpp:35-58
    ScopedSeconds t(secondsDiis);
    double est = 0;
    if (d.DiisStep(0, &est)) {
      lastErrorEst = est;
      used = true;
    }
  } else {
    lastErrorEst = 0;
  }
  eigenvals.resize(n);
  d.Diagonalize(0, occupied, 2.0, eigenvals.data());
  double trace_ph = 0, change2 = 0;
  d.EnergyAndChange(0, &trace_ph, &change2);
  // CalculateEnergy (RestrictedHartreeFock.cpp:209-249)
  HOMOEnergy = eigenvals[nrOccupiedLevels - 1];
  totalEnergy = 0.5 * trace_ph + occupied_sum(eigenvals, occupied) + nuclearRepulsionEnergy;
  d.UpdateDensity(0, used, alpha);
  if (!inCalculate) SyncFromDevice();
  return std::sqrt(change2);
}

hfgpu::Vector3D RestrictedHartreeFock::GetMoment() const {
  return electronic_moment(GetNuclearMoment(), DensityMatrix, nullptr, momentX, momentY, momentZ);
}

double RestrictedHartreeFock::CalculateMp2Energy() {
  const int n = numberOfOrbitals;
  if (!inited || (int)C.rows() != n || (int)eigenvals.size() != n || nrOccupiedLevels >= (unsigned)n) return mp2Energy = 0;
  check_engine(hfg_mp2_rhf(integralsRepository.engine(), C.data(), eigenvals.data(), (int32_t)nrOccupiedLevels, &mp2Energy),
               "hfg_mp2_rhf");
  return mp2Energy;
}

hfgpu::Vector3D UnrestrictedHartreeFock::GetMoment() const {
  return electronic_moment(GetNuclearMoment(), DensityMatrixPlus, &DensityMatrixMinus, momentX, momentY, momentZ);
}

double UnrestrictedHartreeFock::CalculateMp2Energy() {
  const int n = numberOfOrbitals;
  if (!inited || (int)Cplus.rows() != n || (int)Cminus.rows() != n || (int)eigenvalsplus.size() != n ||
      (int)eigenvalsminus.size() != n)
    return mp2Energy = 0;
  check_engine(hfg_mp2_uhf(integralsRepository.engine(), Cplus.data(), eigenvalsplus.data(),
                           (int32_t)nrOccupiedLevelsPlus, Cminus.data(), eigenvalsminus.data(),
                           (int32_t)nrOccupiedLevelsMinus, &mp2Energy),
               "hfg_mp2_uhf");
  return mp2Energy;
}

void UnrestrictedHartreeFock::Init(Systems::Molecule *molecule) {
  HartreeFockAlgorithm::Init(molecule);
  DensityMatrixPlus = Matrix::Zero(h.rows(), h.cols());
  DensityMatrixMinus = Matrix::Zero(h.rows(), h.cols());
  diisPlus = Diis();
  diisMinus = Diis();
  // UnrestrictedHartreeFock.cpp:29-56
  const unsigned el = molecule->ElectronsNumber();
  nrOccupiedLevelsMinus = el / 2;
  nrOccupiedLevelsPlus = el - nrOccupiedLevelsMinus;
  if (molecule->alphaElectrons > 0 || molecule->betaElectrons > 0) {
    nrOccupiedLevelsPlus = molecule->alphaElectrons;
    nrOccupiedLevelsMinus = molecule->betaElectrons;
  }
  const unsigned n = (unsigned)numberOfOrbitals;
  if (nrOccupiedLevelsMinus + nrOccupiedLevelsPlus > 2 * n) nrOccupiedLevelsMinus = nrOccupiedLevelsPlus = n;
  if (nrOccupiedLevelsPlus > n) {
    nrOccupiedLevelsMinus += nrOccupiedLevelsPlus - n;
    nrOccupiedLevelsPlus = n;
  }
  if (nrOccupiedLevelsMinus > n) nrOccupiedLevelsMinus = n;
  occupiedPlus.assign(nrOccupiedLevelsPlus, true);
  occupiedMinus.assign(nrOccupiedLevelsMinus, true);
  device_.reset();
  Device().ResetDiis();
}

void UnrestrictedHartreeFock::SyncToDevice() {
  Device().SetDensity(0, DensityMatrixPlus.data());
  Device().SetDensity(1, DensityMatrixMinus.data());
}

void UnrestrictedHartreeFock::SyncFromDevice() {
  const int n = numberOfOrbitals;
  DensityMatrixPlus.resize(n, n);
  DensityMatrixMinus.resize(n, n);
  Cplus.resize(n, n);
  Cminus.resize(n, n);
  Device().CopyOut(0, DensityMatrixPlus.data(), Cplus.data());
  Device().CopyOut(1, DensityMatrixMinus.data(), Cminus.data());
}

// UnrestrictedHartreeFock::Step (UnrestrictedHartreeFock.cpp:87-191) on the
// device; the Fock matrices are not symmetrised, as in the reference.
double UnrestrictedHartreeFock::Step(int iter) {
  hfgpu::detail::DeviceScf &d = Device();
  if (!inCalculate) SyncToDevice();
  const int n = numberOfOrbitals;
  if (iter == 0) {  // UnrestrictedHartreeFock.cpp:199-222
    Matrix Fp = guess_fock(h, overlap, initGuess);
    Matrix Fm = Fp;
    if (addAsymmetry && n > 1) {
      Fp(0, 1) += asymmetry;
      Fp(1, 0) = Fp(0, 1);
    }
    d.SetFock(0, Fp.data());
    d.SetFock(1, Fm.data());
  } else {
    const auto t0 = std::chrono::steady_clock::now();
    check_engine(hfg_fock_uhf_device(integralsRepository.engine(), d.density(0), d.density(1), d.g_buffer(0),
                                     d.g_buffer(1), d.stream()),
                 "hfg_fock_uhf_device");
    if (shardCount > 1) {
      allReduce(d.g_buffer(0), (size_t)numberOfOrbitals * numberOfOrbitals, d.stream());
      allReduce(d.g_buffer(1), (size_t)numberOfOrbitals * numberOfOrbitals, d.stream());
    }
    AccountDevice(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    d.FockFromG(0, d.g_buffer(0), false);
    d.FockFromG(1, d.g_buffer(1), false);
  }
  bool used = false;
  if (UseDIIS && iter && iter < maxDIISiterations) {  // UnrestrictedHartreeFock.cpp:62-84
    ScopedSeconds t(secondsDiis);
    double ep = 0, em = 0;
    const bool plus = d.DiisStep(0, &ep);
    if (d.DiisStep(1, &em) && plus) {
      lastErrorEst = em + ep;
      used = true;
    }
  } else {
    lastErrorEst = 0;
  }
  eigenvalsplus.resize(n);
  eigenvalsminus.resize(n);
  d.Diagonalize(0, occupiedPlus, 1.0, eigenvalsplus.data());
  d.Diagonalize(1, occupiedMinus, 1.0, eigenvalsminus.data());
  double tp = 0, tm = 0, cp = 0, cm = 0;
  d.EnergyAndChange(0, &tp, &cp);
  d.EnergyAndChange(1, &tm, &cm);
  // CalculateEnergy (UnrestrictedHartreeFock.cpp:246-293)
  const double e = tp + tm + occupied_sum(eigenvalsplus, occupiedPlus) + occupied_sum(eigenvalsminus, occupiedMinus);
  HOMOEnergy = std::max(nrOccupiedLevelsPlus ? eigenvalsplus[nrOccupiedLevelsPlus - 1] : 0.0,
                        nrOccupiedLevelsMinus ? eigenvalsminus[nrOccupiedLevelsMinus - 1] : 0.0);
  totalEnergy = e / 2.0 + nuclearRepulsionEnergy;
  d.UpdateDensity(0, used, alpha);
  d.UpdateDensity(1, used, alpha);
  if (!inCalculate) SyncFromDevice();
  return std::sqrt(cp + cm);
}

}  // namespace HartreeFock

// ===========================================================================
// driver C ABI (include/hfgpu_driver.h)
// ===========================================================================
namespace {
thread_local std::string g_driver_error;

Systems::Molecule build_molecule(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz) {
  Chemistry::Basis basis;
  basis.Load(basis_path);
  Systems::Molecule mol;
  for (int a = 0; a < natoms; ++a) {
    bool found = false;
    for (const auto &b : basis.atoms)
      if ((int)b.Z == Z[a]) {
        mol.atoms.push_back(b);
        mol.atoms.back().position = {xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]};
        found = true;
        break;
      }
    if (!found) throw std::invalid_argument("basis has no element Z=" + std::to_string(Z[a]));
  }
  return mol;
}
}  // namespace

namespace hfgpu {

hfg_status run_scf(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                   const hfd_scf_opts *opts, hfd_scf_result *result, double *density, int64_t density_count,
                   const std::function<void(std::atomic_bool *)> &on_algorithm, std::string *error) {
  if (!basis_path || natoms <= 0 || !Z || !xyz || !opts || !result) return HFG_INVALID_ARG;
  try {
    Systems::Molecule mol = build_molecule(basis_path, natoms, Z, xyz);
    mol.alphaElectrons = (unsigned)opts->alpha_electrons;
    mol.betaElectrons = (unsigned)opts->beta_electrons;
    mol.ElectricField = {opts->electric_field[0], opts->electric_field[1], opts->electric_field[2]};
    mol.Init();
    std::unique_ptr<HartreeFock::HartreeFockAlgorithm> algo;
    const int iters = opts->max_iterations > 0 ? opts->max_iterations : 3000;
    if (opts->unrestricted) algo.reset(new HartreeFock::UnrestrictedHartreeFock(iters));
    else algo.reset(new HartreeFock::RestrictedHartreeFock(iters));
    algo->alpha = opts->alpha;
    algo->initGuess = opts->init_guess;
    algo->UseDIIS = opts->use_diis != 0;
    algo->normalIterAfterDIIS = opts->post_diis;
    algo->integralsRepository.options.eri_convention = opts->eri_convention;
    algo->integralsRepository.options.schwarz_threshold = opts->schwarz_threshold;
    algo->storedIntegralsBudget = 0;  // direct SCF: no stored table needed
    algo->mixedCutoff = opts->mixed_cutoff;
    algo->mixedSwitchEnergy = opts->mixed_switch_energy;
    algo->fp64FinalIterations = opts->fp64_final_iterations;
    algo->mixedSwitchDensity = opts->mixed_switch_density;
    algo->mixedSwitchDiis = opts->mixed_switch_diis;
    algo->fp64FinalConverge = opts->fp64_final_converge != 0;
    algo->stopAtPrecisionTest = opts->stop_at_precision_test != 0;
    algo->incrementalFock = opts->incremental != 0;
    algo->traceIterations = opts->trace != 0;
    algo->concurrentClasses = opts->concurrent_classes >= 1;
    if (opts->shard_count > 1) {
      if (!opts->allreduce) throw std::invalid_argument("shard_count > 1 needs an allreduce callback");
      algo->shardRank = opts->shard_rank;
      algo->shardCount = opts->shard_count;
      const hfd_allreduce_fn fn = opts->allreduce;
      void *user = opts->allreduce_user;
      algo->allReduce = [fn, user](double *g, size_t count, void *stream) { fn(g, (int64_t)count, stream, user); };
    }
    algo->cudaGraphs = opts->concurrent_classes >= 2;
    // the hook sees the terminate flag for the algorithm's whole life
    struct Publish {
      const std::function<void(std::atomic_bool *)> &f;
      Publish(const std::function<void(std::atomic_bool *)> &fn, std::atomic_bool *flag) : f(fn) {
        if (f) f(flag);
      }
      ~Publish() {
        if (f) f(nullptr);
      }
    } publish(on_algorithm, &algo->terminate);
    algo->Init(&mol);
    const double e = algo->Calculate();
    std::memset(result, 0, sizeof *result);
    result->energy = e;
    result->homo = algo->HOMOEnergy;
    result->converged = algo->converged ? 1 : 0;
    result->iterations = algo->iterations;
    result->nbf = algo->numberOfOrbitals;
    result->fock_builds = algo->fockBuilds;
    result->fock_ms_total = algo->fockMilliseconds;
    result->fp32_quartets = algo->fp32Quartets;
    result->fp64_quartets = algo->fp64Quartets;
    result->mixed_steps = algo->mixedSteps;
    result->seconds_fock = algo->secondsFock;
    result->seconds_eigen = algo->secondsEigen;
    result->seconds_diis = algo->secondsDiis;
    result->seconds_total = algo->secondsTotal;
    result->seconds_init = algo->secondsInit;
    const hfgpu::Vector3D mu = algo->GetMoment();
    result->dipole[0] = mu.X;
    result->dipole[1] = mu.Y;
    result->dipole[2] = mu.Z;
    if (opts->mp2 && !opts->unrestricted)
      result->mp2_energy = static_cast<HartreeFock::RestrictedHartreeFock *>(algo.get())->CalculateMp2Energy();
    else if (opts->mp2)
      result->mp2_energy = static_cast<HartreeFock::UnrestrictedHartreeFock *>(algo.get())->CalculateMp2Energy();
    const int64_t nn = (int64_t)result->nbf * result->nbf;
    if (density) {
      if (opts->unrestricted) {
        if (density_count < 2 * nn) return HFG_INVALID_ARG;
        auto *u = static_cast<HartreeFock::UnrestrictedHartreeFock *>(algo.get());
        std::memcpy(density, u->DensityMatrixPlus.data(), nn * sizeof(double));
        std::memcpy(density + nn, u->DensityMatrixMinus.data(), nn * sizeof(double));
      } else {
        if (density_count < nn) return HFG_INVALID_ARG;
        auto *r = static_cast<HartreeFock::RestrictedHartreeFock *>(algo.get());
        std::memcpy(density, r->DensityMatrix.data(), nn * sizeof(double));
      }
    }
    return HFG_OK;
  } catch (const std::invalid_argument &ex) {
    if (error) *error = ex.what();
    return HFG_INVALID_ARG;
  } catch (const std::exception &ex) {
    if (error) *error = ex.what();
    return HFG_DEVICE_ERROR;
  }
}



int64_t job_footprint_bytes(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                            bool unrestricted) {
  Systems::Molecule mol = build_molecule(basis_path, natoms, Z, xyz);
  mol.Init();
  const auto &t = mol.shellTable();
  const int64_t ns = (int64_t)t.L.size(), pairs = ns * (ns + 1) / 2;
  int64_t prim_pairs = 0;
  for (int64_t a = 0; a < ns; ++a)
    for (int64_t b = 0; b <= a; ++b) prim_pairs += (int64_t)t.nprim[a] * t.nprim[b];
  const int64_t tasks = pairs * (pairs + 1) / 2 / 32 + pairs;
  const int64_t nn = (int64_t)t.nbf * t.nbf;
  return 16 * tasks + 144 * prim_pairs + 8 * nn * 32 * (unrestricted ? 2 : 1) + (int64_t(16) << 20);
}

void release_driver_thread() { hfd_release_thread(); }

}  // namespace hfgpu

extern "C" {

const char *hfd_last_error(void) { return g_driver_error.c_str(); }

void hfd_release_thread(void) {
  hfgpu::release_thread_state();
  hfg_release_thread();
}

hfg_status hfd_pulay_solve(const double *B, int32_t m1, int32_t batch, double *c) {
  if (!B || !c || m1 < 2 || batch < 0) return HFG_INVALID_ARG;
  const size_t mm = (size_t)m1 * m1;
  std::vector<double> rhs(m1, 0.0);
  rhs[m1 - 1] = 1.0;
  for (int b = 0; b < batch; ++b) {
    const std::vector<double> x =
        hfgpu::detail::pulay_solve(std::vector<double>(B + b * mm, B + (b + 1) * mm), m1, rhs);
    std::copy(x.begin(), x.end(), c + (size_t)b * m1);
  }
  return HFG_OK;
}

void hfd_default_scf_opts(hfd_scf_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->alpha = 0.75;
  o->init_guess = 0.75;
  o->use_diis = 1;
  o->post_diis = 500;
  o->eri_convention = HFG_ERI_REFERENCE;
  o->schwarz_threshold = 1e-12;
  o->mixed_cutoff = 0;
  o->mixed_switch_energy = 1e-7;
  o->mixed_switch_density = 1e-7;
  o->mixed_switch_diis = 1e-6;
  o->fp64_final_iterations = 2;
  o->fp64_final_converge = 0;
  o->incremental = 0;
  o->trace = 0;
}

hfg_status hfd_scf(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                   const hfd_scf_opts *opts, hfd_scf_result *result, double *density, int64_t density_count) {
  return hfgpu::run_scf(basis_path, natoms, Z, xyz, opts, result, density, density_count, {}, &g_driver_error);
}

hfg_status hfd_one_electron(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz, double *S,
                            double *h, int64_t capacity, int32_t *nbf) {
  if (!basis_path || natoms <= 0 || !Z || !xyz || !nbf) return HFG_INVALID_ARG;
  try {
    Systems::Molecule mol = build_molecule(basis_path, natoms, Z, xyz);
    mol.Init();
    GaussianIntegrals::IntegralsRepository repo(&mol);
    hfgpu::Matrix s, t, v;
    repo.OneElectron(s, t, v);
    const int n = (int)mol.shellTable().nbf;
    *nbf = n;
    if (capacity < (int64_t)n * n) return HFG_INVALID_ARG;
    for (int x = 0; x < n * n; ++x) {
      if (S) S[x] = s.data()[x];
      if (h) h[x] = t.data()[x] + v.data()[x];
    }
    return HFG_OK;
  } catch (const std::exception &ex) {
    g_driver_error = ex.what();
    return HFG_INVALID_ARG;
  }
}

hfg_status hfd_load_xyz(const char *xyz_path, const char *basis_path, int32_t cap, int32_t *natoms, int32_t *Z,
                        double *xyz, int32_t *nbf) {
  if (!xyz_path || !basis_path || !natoms || !nbf) return HFG_INVALID_ARG;
  try {
    Chemistry::Basis basis;
    basis.Load(basis_path);
    Systems::Molecule mol;
    if (!mol.LoadXYZ(xyz_path, basis)) {
      g_driver_error = std::string("LoadXYZ failed for ") + xyz_path;
      return HFG_INVALID_ARG;
    }
    *natoms = (int32_t)mol.atoms.size();
    *nbf = (int32_t)mol.CountNumberOfContractedGaussians();
    for (int32_t i = 0; i < *natoms && i < cap; ++i) {
      if (Z) Z[i] = (int32_t)mol.atoms[i].Z;
      if (xyz) {
        xyz[3 * i] = mol.atoms[i].position.X;
        xyz[3 * i + 1] = mol.atoms[i].position.Y;
        xyz[3 * i + 2] = mol.atoms[i].position.Z;
      }
    }
    return HFG_OK;
  } catch (const std::exception &ex) {
    g_driver_error = ex.what();
    return HFG_INVALID_ARG;
  }
}

}  // extern "C"
