// Autotuner: picks launch shapes (integral-class block shapes, GEMM tiles,
// split counts) by timing the candidates on the device the first time a
// shape key is met, and remembers the fastest for the rest of the process
// (and across processes through the file named by TINYSCF_TUNE_FILE).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace tscf {

bool tune_enabled();
void tune_set_enabled(bool on);
// cached choice for key, or -1
int tune_lookup(const std::string &key);
// time run(c) for every candidate on stream s (one warm-up, `reps` timed
// launches each), store and return the fastest; every candidate must leave
// the same results behind, so the last run's output stands
int tune_run(const std::string &key, const std::vector<int> &cands, const std::function<void(int)> &run,
             cudaStream_t s, int reps = 2);
std::string tune_report();

}  // namespace tscf
