// sidr_host.hpp -- host-side preparation for the evaluator: instance lookup
// tables, the z-statistics, and the rule compiler.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "sidr_internal.hpp"

namespace sidr {

struct HostInstance {
    int n = 0, m = 0, nw = 0;
    double tmax = 0.0;
    std::vector<double> scores, durations, open_t, close_t, d2d, dist;  // SimData arrays
    std::vector<double> F, G, R, P1, P0;                                 // lookup tables
    std::vector<uint32_t> zlt, zle;
    std::vector<double> FR, GD, DP;                                      // neighbour-major
    std::vector<double> CU;                                              // per customer
    std::vector<double> TK;                                              // ATRISK step functions:
    std::vector<uint8_t> TC;                                             // switch points, codes
    int ns = 0;                                                          // sorted row stride
    std::vector<int16_t> ord;                                            // sorted lists
    std::vector<double> sF, sG;
    std::vector<double> bF, bG;                                          // chunk maxima
    std::vector<int32_t> cnt_pos, cnt_gm1;
};

// Validates the SimData arrays (finite, n in range) and builds the tables
// described in sidr_internal.hpp.  Returns an empty string or the error text.
// With tables=false only the arrays are validated and copied (enough for
// host_zstats).
std::string build_instance(int n, int m, double tmax, const double* scores,
                           const double* durations, const double* open_t, const double* close_t,
                           const double* dist, const double* d2d, HostInstance& out,
                           bool tables = true);

// ATRISK's step-function table against the classification it stands for: at
// f = 0, at each switch point and its two neighbours, and at random f in
// [0, 2 tmax), every pair's table outcome other than "classify in full" must
// equal the classification.  Counts the checks and the mismatches.
void atrisk_table_check(const HostInstance& h, int seed, long long& checked, long long& bad);

// zp_of / zstats on the host (engine/sim_host.hpp:96-105,
// engine/sim_core.hpp:277-312).
void host_zstats(const HostInstance& hi, double zp[10]);

// One rule compiled for the kernel.
struct CompiledRule {
    std::vector<uint32_t> prog;
    std::vector<double> consts;
    std::vector<uint8_t> slots;
    int K = 0, D = 0, res = 0, reach_k = 0;
    uint32_t need = 0;
    uint64_t explore = 0;
};

// Validates one post-order rule (engine/vocab.hpp:99-126 encoding) against the
// interpreter's contract -- opcodes in {-2,-1,0..6}, slots < 61, no stack
// underflow, stack depth <= 32, exactly one value left -- and compiles it
// under `mask` (61 flags).  Returns an empty string or the error text.
// all_active_rows: rows 0.. hold every slot active under the mask (ascending,
// the constants C1..C5 excepted) whether the rule reads it or not -- the
// terminal table a decision-situation capture records.
std::string compile_rule(const int32_t* ops, const int32_t* args, int len, const int64_t* mask,
                         CompiledRule& out, bool all_active_rows = false);

// Slot activity under a mask, as pick_best assigns terms[] (engine/sim_core.hpp:
// 84-197): slots 0-9 always; 11 under mask 11 or 33; 14 under 14 or 32; 30
// under 30 or 34; every other slot under its own flag.
bool slot_active(int slot, const int64_t* mask);

// Sets the text sidr_last_error() returns on this thread (the host drivers'
// failures share the C-ABI's error slot).
void set_last_error(const std::string& msg);

}  // namespace sidr
