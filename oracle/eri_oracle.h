/* CPU oracle for the ERI / Fock-build path.  TEST INFRASTRUCTURE ONLY:
 * imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * as the checker; the product library never links it.
 *
 * A plain-C restatement of the reference's algorithm, function by function
 * (file:line citations are to aromanro/HartreeFock, HartreeFock/ directory).
 * Parity pinned against the reference itself, compiled headless by
 * oracle/Makefile into oracle/_ref/ref_driver, and against the golden
 * fixtures that driver wrote under tests/golden/.
 */
#ifndef HF_ERI_ORACLE_H
#define HF_ERI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One contracted Cartesian function, as the reference's
 * ContractedGaussianOrbital (ContractedGaussianOrbital.h:11-31): centre,
 * Cartesian exponents (l,m,n), molecule-wide function ID and shell ID
 * (Molecule.cpp:41-72), and a slice of the primitive arrays. */
typedef struct {
  double center[3];
  int l, m, n;
  int id;       /* contracted ID, running over all functions */
  int shell_id; /* shared by the s and p parts of an SP shell */
  int prim_offset;
  int nprim;
} orc_function;

/* Primitive: exponent, contraction coefficient and per-component
 * normalisation (GaussianOrbital.cpp:25-30, set at basis load
 * Basis.cpp:77-78), kept apart because the reference multiplies them in the
 * order N1 N2 N3 N4 c1 c2 c3 c4 (IntegralsRepository.cpp:405-406). */
typedef struct {
  double alpha;
  double coef;
  double norm;
} orc_primitive;

/* BoysFunction::operator() (BoysFunction.cpp:7-25) with
 * MathUtils::IncompleteGamma (MathUtils.h:163-200). */
double orc_boys_single(double m, double x);
/* BoysFunctions::GenerateBoysFunctions (BoysFunctions.cpp:10-25): F_maxM by
 * orc_boys_single, then downward recursion with exp(-T). */
void orc_boys(int max_m, double T, double *out);

/* IntegralsRepository::getElectronElectron(contracted x4)
 * (IntegralsRepository.cpp:372-433) for function indices i,j,k,l;
 * `max_boys_m` = 4 * Lmax(molecule) + 1 (IntegralsRepository.cpp:334-337).
 * exact_et != 0 computes every electron-transfer row (the true integral);
 * 0 keeps the reference's row range (GaussianTwoElectrons.cpp:162). */
double orc_eri(const orc_function *f, const orc_primitive *p, int i, int j, int k, int l, int max_boys_m,
               int exact_et);

/* Packed 8-fold table, index T(T(i,j),T(k,l)), T(a,b)=max(max+1)/2+min
 * (IntegralsRepository.h:151-162), for all ij >= kl.  OpenMP over i. */
int64_t orc_packed_size(int n);
void orc_eri_packed(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                    double *out);

/* (ij|ij) for every function pair i >= j, at index i(i+1)/2 + j. */
void orc_eri_diagonal(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                      double *out);

/* RestrictedHartreeFock::InitFockMatrix two-electron part
 * (RestrictedHartreeFock.cpp:189-200): G_ij = sum_kl P_kl[(ij|kl) - 1/2 (il|kj)]. */
void orc_g_rhf(int n, const double *packed, const double *P, double *G);
/* Selected rows of the same G, evaluated through orc_eri without a stored
 * table (large molecules): out[r][j] = G_{rows[r], j}. */
void orc_g_rhf_rows(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                    const double *P, const int *rows, int nrows, double *out);
/* UnrestrictedHartreeFock::InitFockMatrices (UnrestrictedHartreeFock.cpp:225-238). */
void orc_g_uhf(int n, const double *packed, const double *Pa, const double *Pb, double *Ga, double *Gb);

/* One-electron matrices (QuantumMatrix.cpp:34-155 through
 * IntegralsRepository.cpp:34-321): overlap, kinetic, nuclear attraction
 * (-sum_A Z_A V_A).  Row-major n x n. */
void orc_one_electron(int n, const orc_function *f, const orc_primitive *p, int natoms, const double *atom_xyz,
                      const int *atom_z, int max_boys_m, double *S, double *T, double *V);

#ifdef __cplusplus
}
#endif
#endif
