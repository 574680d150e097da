// Host-side CNF storage and device packing for the AnalogSAT B200 path.
//
// HostProblem mirrors analogsat::SatProblem (AnalogSAT/problem/SatProblem.{h,cpp}):
// literals are stored flat with per-clause start/length, zero literals are
// filtered, empty clauses are dropped, N = max |literal| and K = max clause length
// (SatProblem.cpp:38-95).
//
// PackedProblem is the device layout of one instance.
//  * Variables are renumbered internally by decreasing degree (number of clause
//    occurrences): perm[v] = public 0-based index of internal variable v, iperm is
//    its inverse.  Groups of 32 consecutive internal variables ("slices") then have
//    nearly equal degrees, so the SELL layout below carries little padding.
//  * Contribution slots (SELL-32): slice g owns rows [srow[g], srow[g+1]) of 32
//    slots; slot (row r, lane l) holds the r-th clause contribution to internal
//    variable 32g+l, rows ordered by (clause, slot) -- the order in which the
//    reference accumulates ds_i (AnalogSAT/cpu_sat/CpuSat.cpp:203-236), so FP64 sums
//    are bit-identical.  Slots past a variable's degree stay 0.
//  * Literal words lit[q * mp + m] (clause m, slot q < k, clause stride mp = M
//    rounded up to 32), one uint32 each:
//        bit 31     negated literal
//        bits 16-30 internal variable index
//        bits 0-15  contribution slot of this literal
//    Slots past a clause's length hold the sentinel word (var = N, slot = nslots):
//    the sentinel spin is held at -1, so each contributes the factor 2 exactly like
//    the reference's zero padding against its constant FALSE slot
//    (CpuSat.cpp:214-215), and its contribution lands in the never-read trash slot
//    nslots, so the kernels store unconditionally.
//    This "compact" encoding needs N < 32768 and at most 65535 slots.  The "wide"
//    encoding (litw: sign << 31 | variable, slotw: slot) has no such limits and is
//    used by the global-storage kernels for larger instances.
//  * Clause order: internally, clauses are regrouped so that the 32 clauses a warp
//    handles together touch 32 different shared-memory banks in each literal slot
//    (the bank of a literal is its internal variable index mod 32, for both the spin
//    gather and the contribution store).  cperm[m] = public clause of internal
//    clause m, icperm is its inverse.  With permute_literals the literals inside a
//    clause may also be reordered for this (FP32 packing only: FP64 keeps the
//    reference's product order to stay bit-identical).  The contribution slots
//    keep the public (clause, literal) order either way.
//  * Pair layout (kPackF32Pair): for the kernel that holds two states per shared
//    array element (float2).  A 64-bit shared access is served per half-warp, and a
//    float2 at index v sits in bank pair v mod 16, so the grouping asks instead that
//    each 16-lane half of a warp touches 16 different bank pairs in every literal
//    slot, and that the 32 clauses of a warp have 32 different public indices mod 32
//    (that kernel reads and writes a_m in place in the public layout).
#pragma once

#include <cstdint>
#include <cstdio>
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
    // The same on an empty problem for zero-free literals (a tokenised CNF body), taking
    // over the literal array instead of copying it.
    void set_clauses(std::vector<int32_t>&& literals, const std::vector<int32_t>& lengths);
};

// CnfReader::Read (AnalogSAT/io/CnfReader.cpp:48-141).  Returns false and fills msg on error.
bool read_cnf(const char* path, HostProblem& p, std::string& msg);
// The preamble part of CnfReader::Read (CnfReader.cpp:54-91): skips lines up to the
// "p cnf N M" declaration and leaves f just after M.  Returns false with msg set when
// the declaration is malformed or missing.
bool read_cnf_header(std::FILE* f, int& n, int& m, std::string& msg);
// The clause body (the bytes after the header) read as CnfReader::Read reads it,
// fscanf-style, from memory: the first m zero-terminated clauses (empty ones
// included).  False with msg "expected more literals in file" or "literal out of
// range" at the first read that fails.
bool parse_cnf_body_host(const char* body, size_t len, long long m, std::vector<int32_t>& literals,
                         std::vector<int32_t>& lengths, std::string& msg);
// CnfWriter::Write (AnalogSAT/io/CnfWriter.cpp:49-74).
bool write_cnf(const char* path, const HostProblem& p);

struct PackedProblem {
    int n = 0, m = 0, k = 0;
    int mp = 0;          // clause stride: m rounded up to a multiple of 32
    int nslices = 0;     // ceil(n / 32)
    int nslots = 0;      // srow[nslices] * 32 (slot nslots is the trash slot)
    bool compact = false;
    std::vector<uint32_t> lit;     // [k][mp] compact literal words (empty unless compact)
    std::vector<uint32_t> litw;    // [k][mp] wide literal words: sign << 31 | internal variable
    std::vector<uint32_t> slotw;   // [k][mp] contribution slot of each wide literal
    std::vector<int32_t> srow;     // [nslices + 1]
    std::vector<int32_t> perm;     // internal -> public variable
    std::vector<int32_t> iperm;    // public -> internal variable
    std::vector<int32_t> cperm;    // internal -> public clause
    std::vector<int32_t> icperm;   // public -> internal clause
    int max_degree = 0;
    long bank_wavefronts = 0;      // shared-memory wavefronts of one gather pass (>= 32-clause groups x k)
    // CTDS variant of the instance (ISat implementation and parameters): tanh = 1 is
    // CpuSatTanh with slope q, b the bias coefficient (ISat::Set_B; 0 = off).
    int tanh = 0;
    double q = 1.1, b = 0.0;
    // clause parts of the lean FP32 kernel's global-rows form (0: none) and the slots of
    // the largest part (set by the solver that builds the PartLayout)
    int lean_parts = 0, lean_part_slots = 0;
};

// Clause parts of the lean FP32 solver's global-rows form: the clauses are split by
// public index into `nparts` ranges, each with its own bank-aware warp grouping and
// its own SELL contribution slots (rows of a variable in public clause order), all
// parts sharing one shared-memory slot buffer of max_slots + 1 entries.  The variable
// phase of part p continues each variable's sum from part p - 1, so the sums run in
// the reference's order.  Words are clause-major, internal clause order (parts
// concatenated): bit 31 negated literal, bits 13-29 the slot in its part's buffer,
// bits 0-12 the internal variable (N < 8191; sentinel N, slot = the part's trash slot).
struct PartLayout {
    int nparts = 0;
    int max_slots = 0;               // largest part's slot count (its trash slot excluded)
    std::vector<int32_t> c0;         // [nparts + 1] first internal clause of each part
    std::vector<int32_t> srow;       // [nparts][nslices + 1] SELL row offsets per part
    std::vector<uint16_t> cnt;       // [nparts][n] occurrences of internal variable v in part p
    std::vector<int32_t> cperm;      // internal -> public clause
    std::vector<int32_t> icperm;     // public -> internal clause
    std::vector<uint32_t> words;     // [m][k]
};
// Builds the parts layout of an instance on the variable order of its FP32 packing q;
// false (layout empty) when N >= 8191 or a part has 2^17 slots or more.
bool pack_parts(const HostProblem& p, const PackedProblem& q, int nparts, PartLayout& out);

enum PackMode : int {
    kPackReference = 0,  // reference literal order (FP64, bit-identical products)
    kPackF32 = 1,        // literals may be reordered; 32-lane bank groups
    kPackF32Pair = 2,    // literals may be reordered; 16-lane bank-pair groups + clause banks
};
PackedProblem pack(const HostProblem& p, int mode);

}  // namespace asb
