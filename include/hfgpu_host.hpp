// hfgpu host API -- the reference's C++ surface over the B200 engine.
//
// Same class names, namespaces, public fields and call sequence as
// aromanro/HartreeFock (HartreeFock/ directory) so that a program written
// against the reference keeps compiling:
//
//   Chemistry::Basis basis; basis.Load("6-31g_st.nw");
//   Systems::Molecule mol;  ... mol.atoms.push_back(atom); mol.Init();
//   HartreeFock::RestrictedHartreeFock hf;   // README.md:63-70
//   hf.alpha = 0.5; hf.initGuess = 0; hf.Init(&mol);
//   double e = hf.Calculate();
//
// The two-electron work (Fock builds, stored integral table, single
// integrals) runs on the GPU through the C ABI of hfgpu.h.  The SCF
// iterations run on the same GPU in FP64 (Fock assembly, DIIS,
// orthogonalisation, cuSOLVER eigensolves, densities), with the public
// fields (DensityMatrix, C, eigenvalues, energies) brought back to the host
// at the end of Calculate() or of a Step() called on its own.  The
// one-electron matrices (S, T, V) are computed on the device at Init
// (hfg_one_electron) and S^-1/2 is formed there too.  Matrices are
// row-major (hfgpu::Matrix) instead of Eigen::MatrixXd; element access
// M(i, j) is the same.
#pragma once

#include <atomic>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "hfgpu.h"

namespace hfgpu {
namespace detail {
class DeviceScf;  // device-resident SCF matrices (internal)
}

class Matrix {
 public:
  Matrix() = default;
  Matrix(int r, int c) : r_(r), c_(c), d_((size_t)r * c, 0.0) {}
  static Matrix Zero(int r, int c) { return Matrix(r, c); }
  int rows() const { return r_; }
  int cols() const { return c_; }
  double &operator()(int i, int j) { return d_[(size_t)i * c_ + j]; }
  double operator()(int i, int j) const { return d_[(size_t)i * c_ + j]; }
  double *data() { return d_.data(); }
  const double *data() const { return d_.data(); }
  void resize(int r, int c) {
    r_ = r;
    c_ = c;
    d_.assign((size_t)r * c, 0.0);
  }

 private:
  int r_ = 0, c_ = 0;
  std::vector<double> d_;
};

Matrix operator*(const Matrix &a, const Matrix &b);
Matrix operator+(const Matrix &a, const Matrix &b);
Matrix operator-(const Matrix &a, const Matrix &b);
Matrix operator*(double s, const Matrix &a);
Matrix transpose(const Matrix &a);
// symmetric eigen-decomposition on the GPU (cuSOLVER dsyevd), eigenvalues
// ascending, eigenvectors as columns
void eigh(const Matrix &a, std::vector<double> &w, Matrix &v);

struct Vector3D {
  double X = 0, Y = 0, Z = 0;
};

}  // namespace hfgpu

namespace Orbitals {
// One basis-file shell line: letters ("S", "SP", "D" ...), exponents, and
// one coefficient column per letter (Basis.cpp:52-83).
struct ContractedGaussianShell {
  std::string letters;
  std::vector<double> exponents;
  std::vector<std::vector<double>> coefficients;
  unsigned CountNumberOfContractedGaussians() const;
};
}  // namespace Orbitals

namespace Chemistry {
class Basis;
}

namespace Systems {

class Atom {
 public:
  hfgpu::Vector3D position;
  unsigned int Z = 0;
  unsigned int electronsNumber = 0;
  unsigned int ID = 0;
  explicit Atom(unsigned int z = 0) : Z(z), electronsNumber(z) {}
};

class AtomWithShells : public Atom {
 public:
  std::vector<Orbitals::ContractedGaussianShell> shells;
  explicit AtomWithShells(unsigned int z = 0) : Atom(z) {}
  unsigned CountNumberOfContractedGaussians() const;
  unsigned GetMaxAngularMomentum() const;
};

class Molecule {
 public:
  std::vector<AtomWithShells> atoms;
  unsigned int alphaElectrons = 0;
  unsigned int betaElectrons = 0;
  hfgpu::Vector3D ElectricField;  // Molecule.h:19; enters h as E . moments

  void Init();  // Molecule.cpp:127-140 (occupations)
  unsigned int CountNumberOfContractedGaussians() const;
  unsigned int ElectronsNumber() const;
  unsigned int GetMaxAngularMomentum() const;
  double NuclearRepulsionEnergy() const;
  double NuclearElectricFieldEnergy() const;  // Molecule.cpp:86-95
  // Molecule::LoadXYZ (Molecule.cpp:143-199): count line, comment line,
  // then "<symbol> x y z" per atom (coordinates used as given, bohr)
  bool LoadXYZ(const std::string &fileName, const Chemistry::Basis &basis);

  // engine-side shell table (one entry per shell letter), rebuilt by Init()
  struct ShellTable {
    std::vector<double> center, exponent, coefficient;
    std::vector<int32_t> L, nprim, prim_offset, ao_offset;
    int32_t nbf = 0;
    hfg_shells view() const;
  };
  const ShellTable &shellTable() const { return table_; }

 private:
  bool LoadXYZBody(const std::string &fileName, const Chemistry::Basis &basis);
  ShellTable table_;
};

}  // namespace Systems

namespace Chemistry {
class Basis {
 public:
  std::vector<Systems::AtomWithShells> atoms;
  void Load(const std::string &fileName);  // Basis.cpp:15-84
};
}  // namespace Chemistry

namespace GaussianIntegrals {

class IntegralsRepository {
 public:
  explicit IntegralsRepository(Systems::Molecule *molecule = nullptr);
  ~IntegralsRepository();
  IntegralsRepository(const IntegralsRepository &) = delete;
  IntegralsRepository &operator=(const IntegralsRepository &) = delete;

  void Reset(Systems::Molecule *molecule = nullptr);
  Systems::Molecule *getMolecule() const { return molecule_; }

  // Stored packed table (IntegralsRepository.cpp:566-584), computed on the GPU.
  void CalculateElectronElectronIntegrals();
  bool HasElectronElectronIntegrals() const { return !packed_.empty(); }
  double getElectronElectron(int i, int j, int k, int l) const;  // .h:138-141
  // single contracted integral without the table (.cpp:372-433)
  double getElectronElectronDirect(int i, int j, int k, int l);

  // No-ops kept for source compatibility: the engine has no host-side memo maps.
  void ClearMatricesMaps() {}
  void ClearElectronElectronIntermediaries() {}
  void ClearElectronElectronMaps() {}
  void ClearAllMaps() {}
  void SetUseLotsOfMemory(bool) {}

  // One-electron matrices (QuantumMatrix.cpp:34-155): overlap, kinetic,
  // nuclear attraction; row-major nbf x nbf.
  void OneElectron(hfgpu::Matrix &S, hfgpu::Matrix &T, hfgpu::Matrix &V) const;
  // Dipole moment matrices about the origin (MomentMatrix, QuantumMatrix.cpp:61-98)
  void Moments(hfgpu::Matrix &Mx, hfgpu::Matrix &My, hfgpu::Matrix &Mz) const;

  hfg_ctx *engine();
  hfg_opts options;  // engine options, used at the next Reset/first use

 private:
  Systems::Molecule *molecule_ = nullptr;
  hfg_ctx *ctx_ = nullptr;
  std::vector<double> packed_;
};

// MO integrals for the post-HF consumers (IntegralsRepository.h:190-291).
// getElectronElectron(p, q, r, s, C) = sum C(mu,p) C(nu,q) C(l,r) C(s',s)
// (mu nu | l s'); the first call computes the whole tensor for its C on the
// device (hfg_mo_eri_full) and later calls read it.  Like the reference,
// whose caches are keyed by orbital indices only, later calls with another
// C return the first C's values.
class MolecularOrbitalsIntegralsRepository {
 public:
  explicit MolecularOrbitalsIntegralsRepository(IntegralsRepository &repository) : repo_(repository) {}
  double getElectronElectron(unsigned p, unsigned q, unsigned r, unsigned s, const hfgpu::Matrix &C);

 private:
  IntegralsRepository &repo_;
  int n_ = 0;
  std::vector<double> mo_;
};

// Antisymmetrised spin-orbital integrals for CCSD / CIS
// (SpinOrbitalsElectronElectronIntegralsRepository.cpp:10-52): spin orbital
// p is spatial orbital p / 2 with spin p % 2, and
// (p, q, r, s) = (p/2 r/2 | q/2 s/2)[same spins p r, q s] - (p/2 s/2 | q/2 r/2)[same spins p s, q r],
// computed on the device (hfg_spin_orbital_eri).
class SpinOrbitalsElectronElectronIntegralsRepository {
 public:
  explicit SpinOrbitalsElectronElectronIntegralsRepository(int numOrbitals);
  SpinOrbitalsElectronElectronIntegralsRepository(int numOrbitals, IntegralsRepository &repository,
                                                  const hfgpu::Matrix &C);
  void Compute(IntegralsRepository &repository, const hfgpu::Matrix &C);
  double operator()(unsigned p, unsigned q, unsigned r, unsigned s) const {
    return t_[((static_cast<size_t>(p) * m_ + q) * m_ + r) * m_ + s];
  }

 private:
  size_t m_ = 0;
  std::vector<double> t_;
};

}  // namespace GaussianIntegrals

namespace HartreeFock {

class HartreeFockAlgorithm {
 public:
  hfgpu::Matrix h;
  int numberOfOrbitals = 0;
  GaussianIntegrals::IntegralsRepository integralsRepository;
  double alpha = 0.75;      // HartreeFockAlgorithm.cpp:10-11
  double initGuess = 0.75;
  std::atomic_bool terminate{false};
  bool converged = false;
  double HOMOEnergy = 0;
  double lastErrorEst = 0;
  bool UseDIIS = true;
  int maxDIISiterations = 1000;
  int normalIterAfterDIIS = 500;
  // engine extension: store the packed table at Init (as the reference
  // always does) only when it fits this many bytes; the Fock builds are
  // direct either way
  size_t storedIntegralsBudget = size_t(1) << 30;
  int iterations = 0;  // steps taken by the last Calculate()

  // Engine extension, no reference counterpart: the precision form of the
  // direct Fock builds (hfgpu.h, hfg_opts).  mixedCutoff > 0 (FP32 below the
  // cutoff) or incrementalFock (FP64) switches it on.  First phase:
  // incremental builds from the density difference with density screening,
  // until |dE| < mixedSwitchEnergy, the density change (rms, as the
  // reference measures it) < mixedSwitchDensity and the DIIS error estimate
  // < mixedSwitchDiis, or the reference's own convergence test passes.  Second phase: fp64FinalIterations full FP64
  // builds from the whole density (density-screened, no history: F is a
  // function of D alone, as in the plain form), after which the SCF counts
  // as converged.  With fp64FinalConverge the second phase instead runs on
  // until the reference's convergence test (Constants.h:6-10) passes too.
  // The incremental phase cannot meet that test itself: every increment
  // adds its screening and FP32 errors to G, which the test's 1e-10-level
  // thresholds resolve.
  double mixedCutoff = 0;
  double mixedSwitchEnergy = 1e-7;
  double mixedSwitchDensity = 1e-7;
  double mixedSwitchDiis = 1e-6;
  int fp64FinalIterations = 2;
  bool fp64FinalConverge = false;
  bool incrementalFock = false;
  // measurement aid: plain FP64 builds throughout, but stopped by the
  // precision form's test (its switch point + fp64FinalIterations steps), for
  // comparing the two forms at equal convergence criteria
  bool stopAtPrecisionTest = false;
  // per-Calculate accounting of the two-electron builds
  double fockMilliseconds = 0;   // device time of all builds
  int fockBuilds = 0;
  int64_t fp32Quartets = 0, fp64Quartets = 0;  // shell quartets evaluated per precision
  int mixedSteps = 0;            // builds of the first (incremental) phase
  // wall-clock split of Calculate (seconds): two-electron builds, the
  // eigensolves, DIIS (error matrices and extrapolation), everything else
  double secondsFock = 0, secondsEigen = 0, secondsDiis = 0, secondsTotal = 0;
  double secondsInit = 0;        // the last Init(): one-electron matrices, engine context, S^-1/2
  bool traceIterations = false;  // one line per step on stderr

  explicit HartreeFockAlgorithm(int iterations = 3000);
  virtual ~HartreeFockAlgorithm();
  virtual void Init(Systems::Molecule *molecule);
  double Calculate();
  virtual double Step(int iter) = 0;
  double GetTotalEnergy() const { return totalEnergy; }
  double GetNuclearElectricFieldEnergy() const { return nuclearElectricFieldEnergy; }
  double GetMP2Energy() const { return mp2Energy; }  // HartreeFockAlgorithm.h:89-92
  // sum_A Z_A R_A (HartreeFockAlgorithm.cpp:234-242)
  hfgpu::Vector3D GetNuclearMoment() const;
  // nuclear moment - sum_ij P_ij <i|r|j> (RestrictedHartreeFock.cpp:319-335,
  // UnrestrictedHartreeFock.cpp:408-424)
  virtual hfgpu::Vector3D GetMoment() const = 0;
  // MomentMatrix: matrix, matrixY, matrixZ (HartreeFockAlgorithm.h)
  hfgpu::Matrix momentX, momentY, momentZ;
  // device execution of the Fock builds (no reference counterpart): CUDA-graph
  // replay of plain builds (for one host thread driving the device: a capture
  // does not mix with other threads' device-wide synchronisation), and a
  // build's classes on concurrent streams.
  bool cudaGraphs = false;
  bool concurrentClasses = false;
  // Sharded Fock builds over several processes / GPUs (no reference
  // counterpart): this algorithm's engine evaluates shard (shardRank,
  // shardCount) of every two-electron build (hfg_set_shard) and allReduce
  // sums the partial G over the shards -- device buffer of `count` doubles,
  // on `stream` -- before F is formed.  Every shard then runs the same SCF
  // algebra on the same G.  shardCount 1: no sharding.
  int shardRank = 0, shardCount = 1;
  std::function<void(double *dG, size_t count, void *stream)> allReduce;
  double mp2Energy = 0;

 protected:
  double totalEnergy;
  double nuclearRepulsionEnergy = 0;
  double nuclearElectricFieldEnergy = 0;
  Systems::Molecule *molecule_ = nullptr;
  hfgpu::Matrix overlap;  // overlapMatrix.matrix
  hfgpu::Matrix V, Vt;    // S^-1/2
  int maxIterations;
  bool inited = false;
  bool fp64Phase = true;  // precision form: the FP32 part is over
  int fp64Steps = 0;      // builds since the switch to FP64
  bool inCalculate = false;  // Step() called from Calculate(): public fields synced at its end
  std::unique_ptr<hfgpu::detail::DeviceScf> device_;
  hfgpu::detail::DeviceScf &Device();
  void AccountDevice(double fock_wall_seconds);
  // copy the public density fields to the device / the device state back
  virtual void SyncToDevice() = 0;
  virtual void SyncFromDevice() = 0;
  bool PrecisionForm() const { return mixedCutoff > 0 || incrementalFock; }
  bool PrecisionCriteria() const { return PrecisionForm() || stopAtPrecisionTest; }
  // convergence decision after a step: `test` is the reference's test
  bool ConvergedAfterStep(bool test, double dE, double rmsD);
  void AccountFockBuild();
  void TraceStep(int iter, double energy, double dE, double rmsD) const;
  void FirstIterations(int &iter, double &curEnergy, double &prevEnergy);
  void SelfConsistentIterations(int &iter, double &curEnergy, double &prevEnergy);
  void NormalIterations(int &iter, double &curEnergy, double &prevEnergy);
};

class Diis {
 public:
  bool AddValueAndError(const hfgpu::Matrix &value, const hfgpu::Matrix &error);
  double Estimate(hfgpu::Matrix &value) const;

 private:
  std::vector<hfgpu::Matrix> errors_, values_;
};

class RestrictedHartreeFock : public HartreeFockAlgorithm {
 public:
  hfgpu::Matrix DensityMatrix;
  unsigned int nrOccupiedLevels = 0;
  std::vector<bool> occupied;
  std::vector<double> eigenvals;
  hfgpu::Matrix C;
  explicit RestrictedHartreeFock(int iterations = 3000) : HartreeFockAlgorithm(iterations) {}
  void Init(Systems::Molecule *molecule) override;
  double Step(int iter) override;
  // RestrictedHartreeFock.cpp:251-288, after Calculate(): the (ia|jb)
  // block by one device AO->MO transform (hfg_mp2_rhf)
  double CalculateMp2Energy();
  hfgpu::Vector3D GetMoment() const override;

 protected:
  void SyncToDevice() override;
  void SyncFromDevice() override;

 private:
  Diis diis;  // host DIIS object kept for source compatibility; the SCF's DIIS runs on the device
};

class UnrestrictedHartreeFock : public HartreeFockAlgorithm {
 public:
  hfgpu::Matrix DensityMatrixPlus, DensityMatrixMinus;
  unsigned int nrOccupiedLevelsPlus = 0, nrOccupiedLevelsMinus = 0;
  std::vector<bool> occupiedPlus, occupiedMinus;
  std::vector<double> eigenvalsplus, eigenvalsminus;
  hfgpu::Matrix Cplus, Cminus;
  bool addAsymmetry = true;  // UnrestrictedHartreeFock.cpp:9
  double asymmetry = 0.1;
  explicit UnrestrictedHartreeFock(int iterations = 3000) : HartreeFockAlgorithm(iterations) {}
  void Init(Systems::Molecule *molecule) override;
  double Step(int iter) override;
  // UnrestrictedHartreeFock.cpp:295-375, on the device (hfg_mp2_uhf)
  double CalculateMp2Energy();
  hfgpu::Vector3D GetMoment() const override;

 protected:
  void SyncToDevice() override;
  void SyncFromDevice() override;

 private:
  Diis diisPlus, diisMinus;  // kept for source compatibility, see RestrictedHartreeFock
};

}  // namespace HartreeFock
