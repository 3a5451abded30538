// output.cuh -- per-step state output (AllVortexSheets / Snapshot2 records).
#pragma once

#include "../../include/uvlm_b200.h"
#include "common.cuh"

namespace uvlm {

// Device state of a time-stepper at the output point of MainLoop (after the
// solve): wing nodes [num][R+1][C+1][3], circulations [num][R][C], wake
// nodes / circulations in rows [wake_start, wake_start + wake_nodes) of
// sheets PR rows tall.
struct OutputState {
  int num, R, C, PR, wake_start, wake_nodes;
  const double* pos;
  const double* gamma;
  const double* wpos;
  const double* wgamma;
};

struct OutputWriter;

// Opens the files that are named (NULL or "" skips one) and starts the writer.
Error output_open(OutputWriter** out, const char* sheet_path, const char* result_path, int device);
// Snapshot on `st` and hand the state to the writer (waits only while both
// staging slots are busy).
Error output_enqueue(OutputWriter* w, const OutputState& s, double t, cudaStream_t st);
// Waits until every queued record is written.
Error output_flush(OutputWriter* w);
// Flushes, stops the writer and closes the files.
Error output_close(OutputWriter* w);
// The legacy simulator's per-step Snapshot2 (OutputSnapshot2,
// src/simulator/simulator.cpp:118-160), host arrays: container shapes, the
// ring pool with reference nodes (rings0 may be null) and one morphing
// velocity record per bound ring (center [3], segment velocities [4][3],
// freestream [3]).
struct LegacySnapshot {
  int64_t n_containers;
  const int64_t* rows;
  const int64_t* cols;
  const double* chord;
  const double* span;
  int64_t n_rings;
  const double* rings;
  const double* rings0;
  const double* gamma;
  int64_t n_mv;
  const double* mv_center;
  const double* mv_nodes;
  const double* mv_freestream;
};
// One unframed Snapshot2 message, replacing the file at path.
Error output_write_legacy_snapshot2(const char* path, double t, const LegacySnapshot& s);
// One record from host arrays (append or truncate).
Error output_encode_to_file(const char* path, int append, int kind, int num, int rows, int cols, int wake_rows,
                            const double* wing_pos, const double* wing_gamma, const double* wake_pos,
                            const double* wake_gamma, double t);

}  // namespace uvlm
