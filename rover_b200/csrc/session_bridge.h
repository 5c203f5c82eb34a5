// session_bridge.h -- what the lane-protocol session service (sessions.cu)
// takes from the library state kept in calculator.cu.
//
// A session runs for as long as its host keeps it open (one call that
// returns at SHUTDOWN), so it does not hold the library lock: it takes a
// snapshot of the loaded index's device view once, and the library refuses
// to unload or replace that index until the session releases it -- the
// reference's DSP skeleton refuses the same (retrieval_async_dsp_search.c:
// 668-696, g_pure_pq_session_live).
#pragma once

#include <cstdint>

#include "kernels.h"

namespace rover {

enum SessionKind : int {
  kSessionPurePq = 0,   // calculator_retrieval_pure_pq_sqmd_run: the pure-PQ index
  kSessionSqmd = 1,     // calculator_retrieval_expand_sqmd(_run): the legacy SQ index
  kSessionDb = 2,       // calculator_retrieval_search_db: the legacy SQ index; calls may overlap
};
constexpr int kSessionKinds = 3;

struct SessionIndex {
  PqIndexView pq{};        // kSessionPurePq: codes and codebook on the device
  uint8_t pq_uuid[16] = {};
  SqIndexView sq{};        // kSessionSqmd / kSessionDb: L1 codes (and graph) on the device
  int32_t sq_graph_entry = -1;
  int device = 0;          // the device the index lives on
};

// Marks a session of `kind` live and fills `out`; false (with the library's
// last error set) when the index it serves is not loaded or another session
// of that kind is live (DB-pair calls may run side by side).
bool session_acquire(SessionKind kind, SessionIndex* out);
void session_release(SessionKind kind);
// Adds to calculator_rover_launch_count.
void session_count_launches(unsigned n);
// Sets calculator_rover_last_error for the calling thread.
void session_error(const char* fmt, ...);

}  // namespace rover
