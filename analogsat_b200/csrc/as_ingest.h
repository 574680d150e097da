// Ingest on the device: initial conditions generated in HBM, and the clause body of a
// DIMACS CNF file tokenised on the GPU.  Both exist for very large instances, where
// the host side (a state vector of N+M values per trajectory copied in, or a CNF body
// of tens of MB read with fscanf) costs more than the solve setup around it.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace asb {

// Distributions of as_solver_set_random_states.
constexpr int kIcSpinUniform = 0;  // s_i ~ U(-1, 1), a_m = a0
constexpr int kIcReference = 1;    // u ~ U[0, 1) for all N+M values, s = 2u - 1, a = u + 1

// One trajectory of a random-state request: element offset of its public state
// [s_1..s_N, a_1..a_M], N and M.
struct IcTraj {
    long long off;
    int n, m;
};

// Writes the initial states of `traj` (host array, nt entries) into `states` (device,
// float when f64 is false, else double) on `stream`.  The trajectories draw in order
// from one stream: Philox4x64-10 keyed by (seed, 0), draw d is output d%4 of the block
// with counter d/4 + 1, uniform u = (x >> 11) * 2^-53.  Allocates and frees a small
// device table; synchronises.
cudaError_t random_states(void* states, bool f64, const std::vector<IcTraj>& traj, unsigned long long seed,
                          int distribution, double a0, cudaStream_t stream);

// Tokenises the clause body of a DIMACS file -- the len bytes of f after the "p cnf N M"
// header, read and copied to the current device piece by piece -- and returns the
// first m clauses: literals concatenated and clause lengths (empty clauses included).  Same acceptance rules as reading the body
// with fscanf("%ld") followed by a range check: returns false with msg set to
// "expected more literals in file" or "literal out of range" on the first failure
// in reading order (or "read failed" when the file ends early), true with msg
// "read ok" otherwise.  cuda receives the first CUDA error (then the return value is
// false and msg names the call).
bool parse_cnf_body(std::FILE* f, size_t len, long long m, std::vector<int32_t>& literals,
                    std::vector<int32_t>& lengths, std::string& msg, cudaError_t& cuda);

}  // namespace asb
