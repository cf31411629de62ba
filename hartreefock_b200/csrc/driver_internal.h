// Internal interface between the one-call SCF driver (host.cpp) and the
// serving pool (pool.cpp).
#pragma once

#include <atomic>
#include <functional>
#include <string>

#include "../../include/hfgpu_driver.h"

namespace hfgpu {

// hfd_scf's body.  `on_algorithm` (may be empty) receives the running
// algorithm's terminate flag once it exists, and nullptr before the
// algorithm is destroyed; setting the flag stops the SCF between iterations
// (HartreeFockAlgorithm::terminate).  Errors go to *error.
hfg_status run_scf(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                   const hfd_scf_opts *opts, hfd_scf_result *result, double *density, int64_t density_count,
                   const std::function<void(std::atomic_bool *)> &on_algorithm, std::string *error);

// Estimated device bytes of one SCF job: quartet task lists (16 B per task
// of up to 32 ket pairs over the triangle of shell pairs), primitive-pair
// tables (96 B FP64 + 48 B FP32 per primitive pair), ~32 n x n FP64
// matrices per spin (h, S, V, F, P, new P, C, G, work, 2 x 6 DIIS entries,
// the incremental history) and a fixed 16 MiB (Boys table, counters,
// library handles).  Throws std::invalid_argument for an unknown element.
int64_t job_footprint_bytes(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                            bool unrestricted);

// frees the calling thread's cuBLAS / cuSOLVER handles and scratch
void release_driver_thread();

}  // namespace hfgpu
