// Batched dynamic-aperture scan: device argument block and launch interface.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_table.hpp"

namespace stb {

constexpr int kMaxScanSeeds = 1024;

// One seed: its element table and its particle range in the flat arrays.
struct ScanSeed {
  const ElemHeader *hdr;
  const double *pool;
  int nelem;
  int npool_padded;
  long off;  // first slot of this seed
  int cap;   // particles of this seed
  int pad;
};

struct ScanArgs {
  const ScanSeed *seeds;
  int nseed;
  int chunk;  // largest work item (particles); the work list may use smaller ones
  int pack;   // nonzero: items always hold `chunk` particles (few CTAs busy, many warps each)
  int grid;   // resident CTAs of the tracking kernel
  RefConsts ref;
  double *x, *px, *y, *py, *z, *pt;  // flat slot arrays
  int32_t *id;                       // original particle index of each slot
  int32_t *lost_turn, *lost_elem;    // per slot (-1: alive)
  int32_t *live;                     // per seed: live particles occupy slots [off, off+live)
  int32_t *items;                    // work list: (seed, first slot) pairs
  int32_t *n_items, *next_item, *item_chunk;
  int32_t *turn0;                    // device turn counter
  int nturn;                         // turns per block
  double r2;
  int loss_mode;  // see is_lost / loss_mode_for
  int *status;
  int32_t *out_lost_turn, *out_lost_elem;  // by original index
  double *out_x;                           // AoS by original index
  // Optional turn-by-turn record at the start of the line: after turn t
  // (global index, t < tbt_turns) x, px, y, py of particle `id` go to
  // tbt[(t * 4 + k) * ntot + id].
  double *tbt;
  int tbt_turns;
  long ntot;
  // Abort flag in mapped host memory (nonzero: every following turn block
  // of the run tracks nothing and leaves the turn counter alone), and the
  // device flag recording that the current block was skipped.
  const volatile int32_t *abort;
  int32_t *block_skipped;
  // Compaction across many CTAs: windows of kCompactWindow slots per seed
  // (nwin per seed), their live counts, and a staging copy of the slots
  // (six coordinates, then the ids) the survivors are gathered into.
  int nwin;
  int32_t *win_count;  // [nseed * nwin]
  double *stage;       // [6 * ntot]
  int32_t *stage_id;   // [ntot]
};

// Slots per compaction window (one CTA each).
constexpr int kCompactWindow = 1024;

// Loss code written for particles removed by stb_scan_retire (never a turn).
constexpr int32_t kRetiredCode = 0x40000000;

struct ScanVariant {
  bool smem;
  int block;
  int min_blocks;
  const char *name;
};
constexpr int kNumScanVariants = 9;
extern const ScanVariant kScanVariants[kNumScanVariants];

// Sets the kernel attributes of a variant and returns its persistent grid size
// (call outside stream capture).
cudaError_t prepare_scan(int variant, int num_sms, size_t smem, int *grid);
// Work list + tracking + compaction of one turn block (stream-ordered, capturable).
cudaError_t launch_scan_block(const ScanArgs &a, int variant, int grid, size_t smem, cudaStream_t st);
// Outputs for the particles still alive.
cudaError_t launch_scan_finalize(const ScanArgs &a, long max_per_seed, cudaStream_t st);
// Marks the live particles whose original index has mask[id] != 0 as retired
// (removed at the next compaction, output lost_turn = kRetiredCode).
cudaError_t launch_scan_retire(const ScanArgs &a, const uint8_t *mask, long max_per_seed, cudaStream_t st);
// One compaction pass (advances the turn counter by a.nturn).
cudaError_t launch_scan_compact_only(const ScanArgs &a, cudaStream_t st);
// Work list + tracking without compaction (variants 0 and 2 only): particles
// keep their slots, lost ones are skipped by their lost_turn.
cudaError_t launch_scan_track_only(const ScanArgs &a, int variant, int grid, size_t smem, cudaStream_t st);

}  // namespace stb
