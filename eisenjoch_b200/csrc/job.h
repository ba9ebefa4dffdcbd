// job.h -- the resumable placement run (defined in api.cu) as the job
// engine drives it.  Nothing here crosses the C ABI.
#pragma once

#include <cstdint>
#include <string>

#include "eplace_internal.h"

namespace eplace {

struct JobState;

// A run of cfg / opts on context c, writing into res (caller buffers sized
// for c's netlist).  shared_pool: host legaliser threads shared with other
// jobs (nullptr: the context's own pool).
JobState *job_create(eplace_ctx *c, const eplace_cfg &cfg, const eplace_opts &opts, eplace_result *res,
                     Pool *shared_pool);
// Validation, initial placement, device reset, first launches' set-up.
// A job whose start fails (or has no cells) is already done().
eplace_status job_start(JobState *j);
// Advances without waiting (block = false): launches intervals, reads
// finished ones, folds finished legalisations.  Returns whether it did any.
bool job_pump(JobState *j, bool block);
bool job_done(const JobState *j);
// Writes the result; waits for the job's host and device legalisations.
eplace_status job_finish(JobState *j);
void job_destroy(JobState *j);

// Marks a context as sharing its device with other jobs' kernels (split,
// non-cooperative step).
void ctx_set_shared(eplace_ctx *c, bool shared);
// Device bytes a context holds.
uint64_t ctx_device_bytes(const eplace_ctx *c);
int ctx_bins_x(const eplace_ctx *c);
int ctx_bins_y(const eplace_ctx *c);
// An empty context on `device` (stream, scalars); nullptr + *st on failure.
eplace_ctx *ctx_new(int32_t device, eplace_status *st);
// The one-shot entry point's kept contexts: take one of `device` (matching
// bin grid preferred), or give one back (destroyed beyond a small limit).
eplace_ctx *take_kept_context(int32_t device, int bx, int by);
void keep_context(eplace_ctx *c);
// Loads a validated problem into a context (buffers reused, only grow).
eplace_status ctx_load_problem(eplace_ctx *c, HostProblem &&hp);
// Whether the tensor-core transform supports the problem's bin grid.
bool problem_tc_supported(const HostProblem &hp);
// Sets the calling thread's last error (eplace_last_error with ctx NULL).
void set_thread_error(const std::string &m);
// Estimated device bytes of a problem once loaded (admission control):
// problem arrays, solver state, bin maps, DCT matrices and the tensor-core
// planes, pinned rings excluded.
uint64_t problem_device_bytes(const HostProblem &hp);

}  // namespace eplace
