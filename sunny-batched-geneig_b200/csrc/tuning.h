// Per-n schedule selection for the stage kernels.
//
// The reference specialises its kernel per (n, pairs per CTA, block size) with NVRTC
// and picks the block size by probing cuSolverDx or by a timing sweep
// (src/nvrtc/nvrtc_solver.cpp:205-240, 649-925, 1021-1042), caching the cubin in
// process and on disk (:392-597).  Here every kernel is compiled ahead of time for
// sm_100a; a schedule is only the launch shape of each stage.  Suggested mode uses a
// built-in table; autotune mode times each stage's candidates on a synthetic batch,
// validates the winning combination against the suggested schedule's results, and
// memoises it in process and in a versioned, checksummed table file (atomic
// write-then-rename; a corrupt or foreign file is ignored and rewritten).
#pragma once

#include <string>

namespace sbg {

struct Schedule {
    int reduce_threads = 256;   // threads per CTA of k_reduce
    int hetrd_threads = 256;    // threads per CTA of k_hetrd
    int back_threads = 256;     // threads per CTA of k_back
    int ql_warps = 4;           // pairs (warps) per CTA of the QL rotation-application kernel
    int chain_threads = 128;    // pairs (threads) per CTA of the QL scalar-chain kernel
    int refine_threads = 256;   // threads per CTA of k_refine (mixed form)
    bool operator==(const Schedule& o) const {
        return reduce_threads == o.reduce_threads && hetrd_threads == o.hetrd_threads &&
               back_threads == o.back_threads && ql_warps == o.ql_warps &&
               chain_threads == o.chain_threads && refine_threads == o.refine_threads;
    }
};

struct TuneRequest {
    int n = 0;
    int device = 0;
    int precision = 0;
    int force_threads = 0;      // 0 = choose; else 128 or 256 for the CTA-per-pair stages
    int force_ql_warps = 0;     // 0 = choose
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
TuneResult select_schedule(const TuneRequest& req);

// Table file helpers (exposed for tests through the C ABI in tuning_capi).
std::string tuning_cache_dir();
std::string tuning_table_path(int device);
void forget_in_process();
// Message returned by sbg_last_error() on this host thread.
void set_last_error(const std::string& msg);

}  // namespace sbg
