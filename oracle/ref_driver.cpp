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
//   alpha <a> | initguess <g> | diis <0|1> | postdiis <n>   algorithm fields
//   mode eri|rhf|uhf|bench       what to run
//   sample <n> | threads <t>     bench mode: function quartets per thread, threads
//   out <file>                   binary output (eri/rhf/uhf modes)
//
// Output file: repeated records  [u32 name_len][name][u64 count][count f64].
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "Basis.h"
#include "IntegralsRepository.h"
#include "Molecule.h"
#include "RestrictedHartreeFock.h"
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
  std::string basisFile, mode = "eri", outFile;
  double alpha = 0.75, initGuess = 0.75;
  int useDiis = 1, postDiis = 500;
  long sample = 20000;
  int threads = 1;
  unsigned alphaEl = 0, betaEl = 0;
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
    else if (key == "alpha") ls >> alpha;
    else if (key == "initguess") ls >> initGuess;
    else if (key == "diis") ls >> useDiis;
    else if (key == "postdiis") ls >> postDiis;
    else if (key == "mode") ls >> mode;
    else if (key == "sample") ls >> sample;
    else if (key == "threads") ls >> threads;
    else if (key == "out") ls >> outFile;
  }

  Chemistry::Basis basis;
  basis.Load(basisFile);
  if (basis.atoms.empty()) { std::fprintf(stderr, "basis %s did not load\n", basisFile.c_str()); return 2; }

  Systems::Molecule molecule;
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
    if (mode == "rhf") algo.reset(new HartreeFock::RestrictedHartreeFock());
    else algo.reset(new HartreeFock::UnrestrictedHartreeFock());
    algo->alpha = alpha;
    algo->initGuess = initGuess;
    algo->UseDIIS = useDiis != 0;
    algo->normalIterAfterDIIS = postDiis;
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
    // The reference's ERI build walks i, j<=i, k, l<=k with ij<=kl
    // (IntegralsRepository.cpp:484-528) through the public contracted
    // accessor.  Each thread owns its own repository, as each GUI job thread
    // owns its own algorithm (HartreeFockDoc.cpp:372-405), and evaluates
    // `sample` canonical function quartets starting at a thread-dependent row,
    // keeping the primitive and contracted maps as the default
    // useLotsOfMemory mode does (IntegralsRepository.h:184).
    const auto fns = Functions(molecule);
    const long n = static_cast<long>(fns.size());
    std::atomic<long> done{0};
    std::vector<std::thread> pool;
    std::vector<double> sink(static_cast<size_t>(threads), 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t]() {
        GaussianIntegrals::IntegralsRepository repo(&molecule);
        long count = 0;
        double acc = 0;
        long i = (n * t) / std::max(threads, 1);
        for (; count < sample; i = (i + 1) % n) {
          for (long j = 0; j <= i && count < sample; ++j) {
            const long long ij = TwoIndex(i, j);
            for (long k = 0; k < n && count < sample; ++k)
              for (long l = 0; l <= k && count < sample; ++l) {
                if (ij > TwoIndex(k, l)) continue;
                acc += repo.getElectronElectron(fns[static_cast<size_t>(i)], fns[static_cast<size_t>(j)],
                                                fns[static_cast<size_t>(k)], fns[static_cast<size_t>(l)]);
                ++count;
              }
          }
        }
        sink[static_cast<size_t>(t)] = acc;
        done += count;
      });
    for (auto &th : pool) th.join();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double s = 0;
    for (double v : sink) s += v;
    std::printf("{\"quartets\": %ld, \"seconds\": %.6f, \"threads\": %d, \"nbf\": %ld, \"checksum\": %.12e}\n",
                done.load(), secs, threads, n, s);
    return 0;
  }
  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 2;
}
