// Per-n schedule selection for the stage kernels.
//
// The reference specialises its kernel per (n, pairs per CTA, block size) with NVRTC
// and picks the block size by probing cuSolverDx or by a timing sweep
// (src/nvrtc/nvrtc_solver.cpp:205-240, 649-925, 1021-1042), caching the cubin in
// process and on disk (:392-597).  Here every kernel is compiled ahead of time for
// sm_100a; a schedule is the launch shape of each stage: pairs per CTA of the warp-per-pair
// kernels (the reference's batches per block), which column-kernel instantiation and how many
// lanes per column, CTA sizes of the CTA-per-pair and QL kernels.  Suggested mode uses a
// built-in table; autotune mode times each stage's candidates on a synthetic batch,
// validates the winning combination (every pair's info, eigenvalues against the built-in
// schedule's, host residuals of sampled columns), and memoises it in process and in a
// versioned, checksummed table file (atomic write-then-rename; a corrupt or foreign file is
// ignored and rewritten).
#pragma once

#include "kernels.cuh"

#include <string>

namespace sbg {

struct Schedule {
    int hetrd_threads = 256;    // threads per CTA of k_hetrd (66 <= n <= 84)
    int pair_warps = 2;         // pairs (warps) per CTA of k_potrf_warp / k_hetrd_warp / k_hetrd_warp_c64
                                // (n <= 65): the reference's batches per block
    int col_exact = 1;          // exact-n column kernels (k_hegst_col, k_back_col) where they exist
    int back_lanes = 1;         // lanes per column of k_back_col (n <= 56)
    int back_qpass = 1;         // reflectors per pass of k_back_col's Q application (n <= 56): 1 or 2
    int reduce_tc = 0;          // n > 84: the triangular stages on the tensor cores (k_reduce_tc, k_back_tc)
    int ql_warps = 4;           // pairs (warps) per CTA of the QL rotation-application kernel
    int chain_threads = 128;    // pairs (threads) per CTA of the QL scalar-chain kernels
    LaunchShape shape() const {
        LaunchShape l;
        l.threads = hetrd_threads;
        l.pair_warps = pair_warps;
        l.col_exact = col_exact;
        l.back_lanes = back_lanes;
        l.back_qpass = back_qpass;
        l.reduce_tc = reduce_tc;
        return l;
    }
    bool operator==(const Schedule& o) const {
        return hetrd_threads == o.hetrd_threads && pair_warps == o.pair_warps && col_exact == o.col_exact &&
               back_lanes == o.back_lanes && back_qpass == o.back_qpass && ql_warps == o.ql_warps &&
               chain_threads == o.chain_threads && reduce_tc == o.reduce_tc;
    }
};

struct TuneRequest {
    int n = 0;
    int device = 0;
    int precision = 0;
    int force_threads = 0;      // 0 = choose; else 128 or 256 for the CTA-per-pair Householder
    int force_bpb = 0;          // 0 = choose; else pairs per CTA (pair_warps for n <= 65, else ql_warps)
    bool autotune = false;
    int cache_mode = 0;         // SBG_CACHE_*
};

struct TuneResult {
    Schedule sched;
    bool autotuned = false;
    bool sweep_ran = false;
    const char* layer = "builtin";   // builtin | in-process | disk | measured
};

Schedule default_schedule(int n, int precision);
// Whether every kernel of the schedule fits the current device's shared memory for order n.
bool schedule_fits(int n, int precision, const Schedule& s);
TuneResult select_schedule(const TuneRequest& req);

// Table file helpers (exposed for tests through the C ABI in tuning_capi).
std::string tuning_cache_dir();
std::string tuning_table_path(int device);
void forget_in_process();
// Message returned by sbg_last_error() on this host thread.
void set_last_error(const std::string& msg);

}  // namespace sbg
