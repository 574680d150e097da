// Host-side CNF storage and device packing for the AnalogSAT B200 path.
//
// HostProblem mirrors analogsat::SatProblem (AnalogSAT/problem/SatProblem.{h,cpp}):
// literals are stored flat with per-clause start/length, zero literals are
// filtered, empty clauses are dropped, N = max |literal| and K = max clause length
// (SatProblem.cpp:38-95).
//
// PackedProblem is the device layout of one instance:
//   lit[q * mp + m]   packed literal word of clause m, slot q (q < k, m < mp):
//                     bits 0..30 = 0-based variable index, bit 31 = negated.
//                     Slots past a clause's length hold the sentinel variable N,
//                     whose spin is held at -1, so each contributes the factor 2
//                     exactly like the reference's zero padding against its
//                     constant FALSE slot (AnalogSAT/cpu_sat/CpuSat.cpp:214-215).
//   sell              var -> (clause, slot) incidence as SELL-32: variables are
//                     cut into slices of 32; slice g owns rows
//                     [sell_row[g], sell_row[g+1]) of 32 entries, lane l of row r
//                     is the r-th incidence of variable 32g+l, given as the
//                     contribution index q * mp + m, -1 past its degree.  Rows
//                     of a variable are ordered by (clause, slot), which is the
//                     order the reference accumulates ds_i in (CpuSat.cpp:203-236),
//                     so FP64 sums are bit-identical.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace asb {

struct HostProblem {
    int n = 0, m = 0, k = 0;
    std::vector<int32_t> storage;  // flat literals, signed, 1-based
    std::vector<int32_t> start;    // per clause
    std::vector<int32_t> length;   // per clause

    // SatProblem::AddClauses(literals, lengths) (SatProblem.cpp:64-95)
    void add_clauses(const int32_t* literals, const int32_t* lengths, int count);
};

// CnfReader::Read (AnalogSAT/io/CnfReader.cpp:48-141).  Returns false and fills msg on error.
bool read_cnf(const char* path, HostProblem& p, std::string& msg);
// CnfWriter::Write (AnalogSAT/io/CnfWriter.cpp:49-74).
bool write_cnf(const char* path, const HostProblem& p);

struct PackedProblem {
    int n = 0, m = 0, k = 0;
    int mp = 0;         // clause stride: m rounded up to a multiple of 32
    int nslices = 0;    // ceil(n / 32)
    std::vector<uint32_t> lit;       // [k][mp]
    std::vector<int32_t> sell_row;   // [nslices + 1]
    std::vector<int32_t> sell;       // [sell_row[nslices]][32]
    int max_degree = 0;
};

PackedProblem pack(const HostProblem& p);

}  // namespace asb
