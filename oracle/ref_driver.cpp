// Headless driver for the reference's own integral and SCF classes.
//
// Test infrastructure only: it is linked against the reference sources
// compiled unmodified by oracle/Makefile into oracle/_ref and is used to pin
// the oracle restatement and to produce the golden fixtures under
// tests/golden/.  It never ships in the product library.
//
// Input (stdin), one directive per line:
//   basis <file>                 NWChem basis file (Basis::Load, Basis.cpp:15-84)
//   atom <Z> <x> <y> <z>         position in bohr; shells copied from the basis
//                                atom with that Z, as Molecule::LoadXYZ does
//                                (Molecule.cpp:143-199)
//   electrons <alpha> <beta>     optional explicit occupations
//   field <Ex> <Ey> <Ez>         Molecule::ElectricField (enters h, HartreeFockAlgorithm.cpp:38)
//   alpha <a> | initguess <g> | diis <0|1> | postdiis <n>   algorithm fields
//   xyz <file>                   Molecule::LoadXYZ(file, basis) instead of atom lines
//                                (Molecule.cpp:143-199); mode xyz prints the result
//   mode eri|rhf|uhf|bench|xyz   what to run
//   sample <n> | threads <t>     bench mode: function quartets per thread, threads
//   spinorb <0|1>                rhf mode: the RHF C and the spin-orbital tensor
//                                SpinOrbitalsElectronElectronIntegralsRepository
//                                (numberOfOrbitals, integralsRepository, C) after the SCF
//   mp2 <0|1>                    rhf/uhf modes: CalculateMp2Energy() after the SCF
//                                (RestrictedHartreeFock.cpp:251-288,
//                                UnrestrictedHartreeFock.cpp:295-375)
//   lowmem <0|1>                 IntegralsRepository::SetUseLotsOfMemory(!lowmem)
//                                (IntegralsRepository.h:143): clear the
//                                primitive maps per shell, as the GUI's option
//                                does (HartreeFockThread.cpp:31), so large
//                                molecules fit in host memory
//   out <file>                   binary output (eri/rhf/uhf modes)
//
// Output file: repeated records  [u32 name_len][name][u64 count][count f64].
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <cmath>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "Basis.h"
#include "IntegralsRepository.h"
#include "Molecule.h"
#include "RestrictedHartreeFock.h"
#include "SpinOrbitalsElectronElectronIntegralsRepository.h"
#include "UnrestrictedHartreeFock.h"

namespace {

struct Writer {
  std::ofstream f;
  explicit Writer(const std::string &path) : f(path, std::ios::binary) {}
  void put(const std::string &name, const std::vector<double> &v) {
    const uint32_t n = static_cast<uint32_t>(name.size());
    const uint64_t c = v.size();
    f.write(reinterpret_cast<const char *>(&n), sizeof n);
    f.write(name.data(), n);
    f.write(reinterpret_cast<const char *>(&c), sizeof c);
    f.write(reinterpret_cast<const char *>(v.data()), static_cast<std::streamsize>(c * sizeof(double)));
  }
  void put(const std::string &name, const Eigen::MatrixXd &m) {
    std::vector<double> v(static_cast<size_t>(m.rows() * m.cols()));
    for (long i = 0; i < m.rows(); ++i)
      for (long j = 0; j < m.cols(); ++j) v[static_cast<size_t>(i * m.cols() + j)] = m(i, j);  // row-major
    put(name, v);
  }
  void put(const std::string &name, double x) { put(name, std::vector<double>{x}); }
};

// The algorithms with their Step() calls counted (Step is the public
// virtual one SCF iteration, HartreeFockAlgorithm.h:80; Calculate drives it).
struct CountingRhf : HartreeFock::RestrictedHartreeFock {
  int steps = 0;
  double Step(int iter) override { ++steps; return HartreeFock::RestrictedHartreeFock::Step(iter); }
};
struct CountingUhf : HartreeFock::UnrestrictedHartreeFock {
  int steps = 0;
  double Step(int iter) override { ++steps; return HartreeFock::UnrestrictedHartreeFock::Step(iter); }
};

long long TwoIndex(long long i, long long j) { return i < j ? j * (j + 1) / 2 + i : i * (i + 1) / 2 + j; }

// all contracted functions of the molecule, in the repository's walk order
// (atoms -> shells -> basis functions, IntegralsRepository.cpp:566-578)
std::vector<const Orbitals::ContractedGaussianOrbital *> Functions(const Systems::Molecule &m) {
  std::vector<const Orbitals::ContractedGaussianOrbital *> out;
  for (const auto &atom : m.atoms)
    for (const auto &shell : atom.shells)
      for (const auto &orb : shell.basisFunctions) out.push_back(&orb);
  return out;
}

}  // namespace

int main() {
  std::string basisFile, mode = "eri", outFile, xyzFile;
  double alpha = 0.75, initGuess = 0.75;
  int useDiis = 1, postDiis = 500;
  long sample = 20000;
  int threads = 1;
  int lowmem = 0;
  int mp2 = 0;
  int spinorb = 0;
  unsigned alphaEl = 0, betaEl = 0;
  double field[3] = {0, 0, 0};
  struct AtomSpec { unsigned Z; double x, y, z; };
  std::vector<AtomSpec> specs;

  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream ls(line);
    std::string key;
    if (!(ls >> key)) continue;
    if (key == "basis") ls >> basisFile;
    else if (key == "atom") { AtomSpec a{}; ls >> a.Z >> a.x >> a.y >> a.z; specs.push_back(a); }
    else if (key == "electrons") ls >> alphaEl >> betaEl;
    else if (key == "field") ls >> field[0] >> field[1] >> field[2];
    else if (key == "alpha") ls >> alpha;
    else if (key == "initguess") ls >> initGuess;
    else if (key == "diis") ls >> useDiis;
    else if (key == "postdiis") ls >> postDiis;
    else if (key == "mode") ls >> mode;
    else if (key == "sample") ls >> sample;
    else if (key == "threads") ls >> threads;
    else if (key == "lowmem") ls >> lowmem;
    else if (key == "mp2") ls >> mp2;
    else if (key == "spinorb") ls >> spinorb;
    else if (key == "xyz") ls >> xyzFile;
    else if (key == "out") ls >> outFile;
  }

  Chemistry::Basis basis;
  basis.Load(basisFile);
  if (basis.atoms.empty()) { std::fprintf(stderr, "basis %s did not load\n", basisFile.c_str()); return 2; }

  Systems::Molecule molecule;
  if (!xyzFile.empty()) {
    const bool ok = molecule.LoadXYZ(xyzFile, basis);
    if (mode == "xyz") {
      std::printf("{\"ok\": %s, \"atoms\": [", ok ? "true" : "false");
      for (size_t i = 0; ok && i < molecule.atoms.size(); ++i)
        std::printf("%s[%u, %.17g, %.17g, %.17g]", i ? ", " : "", molecule.atoms[i].Z, molecule.atoms[i].position.X,
                    molecule.atoms[i].position.Y, molecule.atoms[i].position.Z);
      std::printf("], \"nbf\": %u}\n", ok ? molecule.CountNumberOfContractedGaussians() : 0u);
      return 0;
    }
    if (!ok) { std::fprintf(stderr, "LoadXYZ failed\n"); return 2; }
  }
  for (const auto &s : specs) {
    bool found = false;
    for (const auto &ba : basis.atoms)
      if (ba.Z == s.Z) {
        molecule.atoms.push_back(ba);
        molecule.atoms.back().position = Vector3D<double>(s.x, s.y, s.z);
        found = true;
        break;
      }
    if (!found) { std::fprintf(stderr, "no basis for Z=%u\n", s.Z); return 2; }
  }
  molecule.alphaElectrons = alphaEl;
  molecule.betaElectrons = betaEl;
  molecule.ElectricField = Vector3D<double>(field[0], field[1], field[2]);
  molecule.Init();

  if (mode == "eri") {
    Writer w(outFile);
    GaussianIntegrals::IntegralsRepository repo(&molecule);
    const auto t0 = std::chrono::steady_clock::now();
    repo.CalculateElectronElectronIntegrals();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const int n = static_cast<int>(molecule.CountNumberOfContractedGaussians());
    std::vector<double> packed(static_cast<size_t>(TwoIndex(TwoIndex(n - 1, n - 1), TwoIndex(n - 1, n - 1)) + 1));
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j)
        for (int k = 0; k < n; ++k)
          for (int l = 0; l <= k; ++l) {
            const long long ij = TwoIndex(i, j), kl = TwoIndex(k, l);
            if (ij < kl) continue;
            packed[static_cast<size_t>(TwoIndex(ij, kl))] = repo.getElectronElectron(i, j, k, l);
          }
    w.put("eri_packed", packed);
    w.put("eri_seconds", secs);
    // one-electron matrices through the same classes HartreeFockAlgorithm::Init uses
    HartreeFock::RestrictedHartreeFock rhf;
    rhf.Init(&molecule);
    w.put("h", rhf.h);
    w.put("enuc", molecule.NuclearRepulsionEnergy());
    w.put("nbf", static_cast<double>(n));
    return 0;
  }

  if (mode == "rhf" || mode == "uhf") {
    Writer w(outFile);
    std::unique_ptr<HartreeFock::HartreeFockAlgorithm> algo;
    CountingRhf *crhf = nullptr;
    CountingUhf *cuhf = nullptr;
    if (mode == "rhf") algo.reset(crhf = new CountingRhf());
    else algo.reset(cuhf = new CountingUhf());
    algo->alpha = alpha;
    algo->initGuess = initGuess;
    algo->UseDIIS = useDiis != 0;
    algo->normalIterAfterDIIS = postDiis;
    algo->integralsRepository.SetUseLotsOfMemory(lowmem == 0);
    const auto t0 = std::chrono::steady_clock::now();
    algo->Init(&molecule);
    const auto t1 = std::chrono::steady_clock::now();
    const double e = algo->Calculate();
    const auto t2 = std::chrono::steady_clock::now();
    w.put("energy", e);
    w.put("converged", algo->converged ? 1.0 : 0.0);
    w.put("homo", algo->HOMOEnergy);
    w.put("init_seconds", std::chrono::duration<double>(t1 - t0).count());
    w.put("scf_seconds", std::chrono::duration<double>(t2 - t1).count());
    w.put("iterations", static_cast<double>(crhf ? crhf->steps : cuhf->steps));
    {
      const Vector3D<double> mu = algo->GetMoment();
      w.put("dipole", std::vector<double>{mu.X, mu.Y, mu.Z});
    }
    if (mp2) w.put("mp2", algo->CalculateMp2Energy());
    if (spinorb && crhf) {
      const int n = crhf->numberOfOrbitals;
      GaussianIntegrals::SpinOrbitalsElectronElectronIntegralsRepository so(n, crhf->integralsRepository, crhf->C);
      std::vector<double> t(static_cast<size_t>(16) * n * n * n * n);
      size_t k = 0;
      for (int p = 0; p < 2 * n; ++p)
        for (int q = 0; q < 2 * n; ++q)
          for (int r = 0; r < 2 * n; ++r)
            for (int s = 0; s < 2 * n; ++s) t[k++] = so(p, q, r, s);
      w.put("C", crhf->C);
      w.put("spin_orbital_eri", t);
    }
    w.put("h", algo->h);
    if (mode == "rhf") {
      auto *r = static_cast<HartreeFock::RestrictedHartreeFock *>(algo.get());
      w.put("density", r->DensityMatrix);
    } else {
      auto *u = static_cast<HartreeFock::UnrestrictedHartreeFock *>(algo.get());
      w.put("density_alpha", u->DensityMatrixPlus);
      w.put("density_beta", u->DensityMatrixMinus);
    }
    return 0;
  }

  if (mode == "bench") {
    // The reference's ERI build evaluates every 8-fold unique function
    // quartet (i >= j, k >= l, ij >= kl; IntegralsRepository.cpp:484-584)
    // through the public contracted accessor.  Each thread owns its own
    // repository, as each GUI job thread owns its own algorithm
    // (HartreeFockDoc.cpp:372-405), and evaluates `sample` quartets drawn
    // uniformly at random from that whole set (seeded per thread), so the
    // measured rate is the build's average over its mix of quartet classes
    // and contraction lengths.  The primitive and contracted maps are kept,
    // as the default useLotsOfMemory mode does (IntegralsRepository.h:184).
    const auto fns = Functions(molecule);
    const long n = static_cast<long>(fns.size());
    const unsigned long long npair = static_cast<unsigned long long>(n) * (n + 1) / 2;
    const unsigned long long nall = npair * (npair + 1) / 2;
    // triangular decode: r -> (hi, lo) with r = hi (hi + 1) / 2 + lo, lo <= hi
    auto untri = [](unsigned long long r, unsigned long long *hi, unsigned long long *lo) {
      unsigned long long h = static_cast<unsigned long long>((std::sqrt(8.0 * static_cast<double>(r) + 1.0) - 1.0) / 2.0);
      while (h * (h + 1) / 2 > r) --h;
      while ((h + 1) * (h + 2) / 2 <= r) ++h;
      *hi = h;
      *lo = r - h * (h + 1) / 2;
    };
    std::atomic<long> done{0};
    std::vector<std::thread> pool;
    std::vector<double> sink(static_cast<size_t>(threads), 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t]() {
        GaussianIntegrals::IntegralsRepository repo(&molecule);
        std::mt19937_64 rng(12345u + 7919u * static_cast<unsigned>(t));
        std::uniform_int_distribution<unsigned long long> pick(0, nall - 1);
        long count = 0;
        double acc = 0;
        for (; count < sample; ++count) {
          unsigned long long ij, kl, i, j, k, l;
          untri(pick(rng), &ij, &kl);
          untri(ij, &i, &j);
          untri(kl, &k, &l);
          acc += repo.getElectronElectron(fns[static_cast<size_t>(i)], fns[static_cast<size_t>(j)],
                                          fns[static_cast<size_t>(k)], fns[static_cast<size_t>(l)]);
        }
        sink[static_cast<size_t>(t)] = acc;
        done += count;
      });
    for (auto &th : pool) th.join();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double s = 0;
    for (double v : sink) s += v;
    std::printf("{\"quartets\": %ld, \"seconds\": %.6f, \"threads\": %d, \"nbf\": %ld, \"unique_quartets\": %llu, "
                "\"sample\": \"uniform\", \"checksum\": %.12e}\n",
                done.load(), secs, threads, n, nall, s);
    return 0;
  }
  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 2;
}
