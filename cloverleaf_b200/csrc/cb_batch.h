// cb_batch.h -- device-side description of a batched ensemble of independent
// decks and the declarations of the persistent ensemble kernel's launchers.
//
// A batch holds many meshes, each laid out exactly as a cb_chunk lays out
// one (cb_chunk.h: same pitch, offset, 19 buffers and tensor maps), each
// with its own gamma, states, dt controls and end time.  One launch of the
// persistent kernel advances every deck from its initial state to its end.
// Each deck has a width w (CTAs, a power of two) and waits in the queue of
// its width, largest first.  The queues are worked widest first: at width W
// the grid is cut into lanes of W consecutive CTAs; a lane takes the next
// deck of the queue (one atomic add by its first CTA, shared at a lane
// barrier), its CTAs share the deck's tiles and meet at a lane barrier
// between the phases, and when the queue is empty the lane splits into the
// lanes of the next width.  No CTA waits for a deck to gather its CTAs, and
// a lane that finishes early goes on with narrower decks.  Every CTA of a
// lane steps through the same control flow (dt, time, step, summaries) with
// identical values, so no control state has to be exchanged besides the dt
// minimum.  A deck's width is fixed by the schedule, so its results do not
// depend on which lane ran it.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "cb_chunk.h"
#include "cb_ops.h"

namespace cb {

constexpr int BATCH_MAX_STATES = 8;
constexpr int BATCH_RECORD = 7;       // summary record: step, time, vol, mass, ie, ke, press
constexpr int BATCH_MAX_LANE = 1024;  // CTAs per lane at most
constexpr int BATCH_VARIANTS = 2;     // tile-shape variants of the kernel (BatchTune)

// Deck status after a run.
enum : int {
  DECK_PENDING = 0,     // not reached (the lane stopped earlier)
  DECK_DONE = 1,        // reached end_time or end_step
  DECK_SMALL_DT = 2,    // dt fell below dtmin (driver/timestep.cpp:96, :104-106)
  DECK_STAGE_FAIL = 3,  // a tile's bulk copy did not arrive within the wait limit
  DECK_SYNC_FAIL = 4,   // a lane barrier gave up (or another lane's did)
};

struct BatchDeck {
  // layout (as cb_create lays out one chunk)
  int nx, ny, off, pitch;
  size_t buf_bytes;           // bytes of each buffer (a multiple of 256)
  void *buf[BATCH_BUF];        // the 15 state fields in field order, then the 4 spares
  const CUtensorMap *maps;     // [BATCH_BUF][NUM_BOX_H], in global memory
  const double *geom_d[NUM_GEOM];
  const void *geom_t[NUM_GEOM];
  const double *rgeom;        // 1 / celldx, 1 / celldy, 1 / vertexdx, 1 / vertexdy
  int geom_len;
  // the deck (driver/definitions.h:227-256 globals that the step reads)
  double gm1;                 // gamma - 1
  int nstates;
  DevState states[BATCH_MAX_STATES];
  double dtinit, dtmin, dtmax, dtrise, end_time;
  int end_step, summary_frequency;
  DtConsts k;
  // records
  double *summaries;          // BATCH_RECORD doubles per record
  int max_summaries;
  double *dt_trace;           // dt of each step
  int max_steps;
  unsigned long long *dt_slots; // 3 reduction slots, rotated by step
  double *partials;           // 5 per CTA of the lane
  // results, written by the lane's first CTA when the deck ends
  int steps, nsummaries, status;
  double time;
};

struct BatchLaunch {
  BatchDeck *decks;
  const int *queue;      // the decks, queue after queue (widest first), each largest first
  const int *level;      // per width k: width | first queue position | decks | first lane slot (4 ints)
  int nlevels;
  unsigned *next;        // next queue position to hand out, per width (zero at launch)
  unsigned *lane_sync;   // barrier counter of each lane slot (zero at launch)
  int *lane_deck;        // the deck a lane took (written by its first CTA), per lane slot
  int *abort;            // set when a barrier wait gives up; ends every lane
  int *err;              // set when a staging wait gives up
};

template <typename T> struct BatchOps {
  // dynamic shared memory of the kernel variant
  static size_t smem_bytes(int variant);
  // resident CTAs per SM of the variant
  static cudaError_t occupancy(int variant, int *per_sm);
  // one launch of the whole ensemble (cooperative: every CTA co-resident)
  static cudaError_t launch(int variant, const BatchLaunch &a, int grid, cudaStream_t s);
};

extern template struct BatchOps<double>;
extern template struct BatchOps<float>;

} // namespace cb
