// The encoder's two-phase tile packer (host code in entropy.cu): phase 1
// turns each superblock's tokens into the range coder's stores with the CDF
// adaptation, phase 2 codes the stores with the cdef_idx literals inserted,
// following phase 1 superblock by superblock from another thread.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <atomic>
#include <vector>

namespace mth {

// Phase 1 runs as kTracers workers per tile.  A CDF's adaptation depends only
// on the symbols coded with it, so the CDF slots are split between the
// workers (slot parity; the raw-bit bools go to worker 0): each worker walks
// every token to count the stores, adapts its own copy of the CDF set and
// writes the stores of its own tokens.
constexpr int kTracers = 2;

// The stores of one tile.  st holds one (fl << 24 | fh << 8 | nms) store per
// token and is sized before phase 1 starts; worker 0 writes sb_end / cdef_at
// per superblock; each worker's `done` passes a superblock once its stores
// there are written (release); `failed` marks a malformed token, after which
// that worker's `done` jumps to the tile's superblock count.
struct TileStores {
  std::vector<uint64_t> st;
  std::vector<uint32_t> sb_end;   // end of each superblock's stores
  std::vector<uint32_t> cdef_at;  // store index of each superblock's read_cdef() point, or UINT32_MAX
  std::atomic<int> done[kTracers] = {};
  std::atomic<bool> failed{false};
};

// Phase 1 over superblocks [0, nsb) of a tile: sbs[i] holds superblock i's
// syntax tokens with 0xFFFFFFFF standing for the next coefficient block, whose
// tokens are toks[offs[k] .. offs[k + 1]) (k from first_coef on);
// cdef_point[i] is the syntax-token index before which read_cdef() falls
// (-1: none).
// `part` (0 .. kTracers - 1) is this worker's share.
void trace_tile_stores(uint8_t base_q_idx, int32_t updating_cdf, const std::vector<uint32_t>* sbs, int nsb,
                       const int32_t* cdef_point, const uint32_t* toks, const uint32_t* offs, size_t first_coef,
                       TileStores* out, int part);

// Phase 2: the coder over the stores of the tile's nsb superblocks, waiting
// for every phase-1 worker as it goes; cdef_idx[i] is coded as a raw cdef_bits-bit literal
// at superblock i's read_cdef() point when cdef_bits > 0.  The tile's bytes
// in *payload (malloc).
int code_tile_stores(TileStores* in, int nsb, int32_t updating_cdf, const uint8_t* cdef_idx, int32_t cdef_bits,
                     uint8_t** payload, size_t* payload_len);

}  // namespace mth
