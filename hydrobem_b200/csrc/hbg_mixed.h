// hbg_mixed.h -- the mixed-precision form (complex64 matrices, tensor-core LU, FP64 refinement).
#pragma once
#include <cstdint>
#include <functional>
#include <vector>

#include "../../include/hydrobem_gpu.h"
#include "hbg_internal.h"

namespace hbg {

// The field points of a problem on the device: P points [P][3] and their statics rows [4][P][N].
struct FieldArgs {
    const double* pts;
    int P;
    const double* stp;
};

// Solve every frequency of one body in the mixed form.  start() queues the statics st (FP64,
// [4][N*N]) on stream s; it is called once the host-side setup (batch sizing, buffers, kernel
// attributes) is done, before the first assembly.  motion: the motion matrices M, C, B_ext (D x D each,
// one after the other, written by the statics stage) when the problem wants motions, else null; field:
// the field points (P = 0: none); fallback: receives the frequencies whose refinement did not converge (or
// whose unpivoted LU met a zero pivot), their outputs left unwritten for the FP64 form.  Returns 0, or an HbStatus with the message in *msg and the frequency in *freq.
int mixed_solve_frequencies(const PanelsView& pv, const double* st, const HbgProblem& pr, const HbgOptions& opt,
                            bool finite, double depth, cudaStream_t s, double* prof, int64_t* launches,
                            const char** msg, int64_t* freq, const std::function<void()>& start,
                            const double* motion, const FieldArgs& field, std::vector<int64_t>* fallback);

int debug_gemm_tf32(int M, int N, int K, const float* A, const float* B, float* C, bool subtract, const char** msg);
int measure_peaks(double* out, const char** msg);
// the mixed LU's groups of systems on side streams for the solves that follow (process-wide; 0: the
// library's rule)
void mixed_lu_groups(int groups);

}  // namespace hbg
