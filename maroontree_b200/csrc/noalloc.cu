// Allocation-free form of the batched 8x8 RDO level (mt_rdo_level8_device_noalloc).
//
// Some hosts cannot hand this library device memory on demand: an encoder
// thread that runs under a fixed GPU-memory budget owned by another
// framework's pool, a real-time path that must not call into the driver's
// allocator (cudaMalloc can synchronise the device and stall other streams),
// or a caller that only owns the buffers of its own inputs and outputs.  For
// them this entry point needs no working storage from the caller and makes no
// allocation of its own: the per-block argmin keys live in one fixed-size
// file-scope device array, and instead of keeping every candidate's result it
// evaluates every candidate for the argmin only, then re-evaluates each
// block's winner (one candidate per block) to fill the output record.
//
// Limits and sharing: at most MT_NOALLOC_MAX_BLOCKS blocks per call (8 bytes
// each, 1 MiB held on every device that loads the library until the process
// exits).  All calls share the one array and it keeps the last call's
// contents; the keys are reset at the start of every call.  Calls whose work
// overlaps on the GPU (different streams, or different host threads without
// ordering) race on the array and must not be issued.
#include <cuda_runtime.h>
#include <stdint.h>

#include "chain8.cuh"

namespace mth {
float scaled_trellis_lambda_host(float dc_q, float lambda0);
}

namespace {

constexpr int kNoAllocThreads = 128;

// Per-block argmin keys of the allocation-free level.
static __device__ __align__(256) unsigned long long g_noalloc_keys[MT_NOALLOC_MAX_BLOCKS];

struct NoAllocArgs {
  mt_chain_params p;
  mt_quant q;
  float trellis_lambda;
  int has_qm;
};

__device__ __forceinline__ bool noalloc_candidate(const mt_block8& bk, const mt_combo& cb, mt_candidate& cd) {
  cd.px = bk.px;
  cd.py = bk.py;
  cd.mode = cb.mode;
  cd.angle_delta = cb.angle_delta;
  cd.tx_type = cb.tx_type;
  cd.flags = (uint8_t)((bk.flags & ~MT_CAND_NO_TRELLIS) | ((cb.flags & MT_COMBO_NO_TRELLIS) ? MT_CAND_NO_TRELLIS : 0));
  cd.dcs_ctx = bk.dcs_ctx;
  cd.skip_ctx = bk.skip_ctx;
  cd.reserved = 0;
  cd.mode_bits = cb.mode <= MT_PAETH_PRED ? bk.mode_bits[cb.mode] : 0.0f;
  cd.extra_bits = cb.bits;
  return true;
}

__device__ __forceinline__ void noalloc_tables(const mt_coef_costs* __restrict__ costs,
                                               const uint8_t* __restrict__ qm_row, int has_qm, mt_coef_costs& sC,
                                               uint8_t* sQm, float* sQs, float* sLut) {
  const float* g = reinterpret_cast<const float*>(costs);
  float* s = reinterpret_cast<float*>(&sC);
  for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
  if (threadIdx.x < 64) {
    const int w = has_qm ? qm_row[threadIdx.x] : 32;
    sQm[threadIdx.x] = (uint8_t)w;
    sQs[threadIdx.x] = mtd::fwd_qm_scale(w);
    sLut[threadIdx.x] = mtd::kCoefRateLut[threadIdx.x];
  }
  __syncthreads();
}

// Pass 1: every (combo, block) candidate, folded into the block's key
// (cost bits << 32 | combo), the same order as the level kernel's argmin.
template <bool VIS>
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_keys_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, NoAllocArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs, const mt_block8* __restrict__ blocks,
    int nblocks, const mt_combo* __restrict__ combos, int ncombos, unsigned long long* __restrict__ keys) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  __shared__ float sLut[64];
  noalloc_tables(costs, qm_row, a.has_qm, sC, sQm, sQs, sLut);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(t / nblocks), b = (int)(t - (long long)c * nblocks);
  if (c >= ncombos) return;
  mt_candidate cd;
  noalloc_candidate(blocks[b], combos[c], cd);
  if (!mtd::cand_ok(cd, a.p.frame_w, a.p.frame_h)) return;
  int32_t store[mtd::kWork8Words];
  mtd::Work8 w{store};
  mt_candidate_result r;
  mtd::chain8_one<VIS>(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
  atomicMin(&keys[b], ((unsigned long long)__float_as_uint(r.cost) << 32) | (unsigned)c);
}

// Pass 2: one thread per block re-evaluates its winning candidate.
template <bool VIS>
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_winner_kernel(
    const uint16_t* __restrict__ src, const uint16_t* __restrict__ rec, NoAllocArgs a,
    const uint8_t* __restrict__ qm_row, const mt_coef_costs* __restrict__ costs, const mt_block8* __restrict__ blocks,
    int nblocks, const mt_combo* __restrict__ combos, const unsigned long long* __restrict__ keys,
    mt_block_best* __restrict__ best) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  __shared__ float sLut[64];
  noalloc_tables(costs, qm_row, a.has_qm, sC, sQm, sQs, sLut);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const unsigned long long k = keys[b];
  mt_block_best o = {};
  if (k == ~0ull) {
    o.combo = -1;
    o.eob = MT_EOB_INVALID;
  } else {
    const int c = (int)(k & 0xffffffffu);
    mt_candidate cd;
    noalloc_candidate(blocks[b], combos[c], cd);
    int32_t store[mtd::kWork8Words];
  mtd::Work8 w{store};
    mt_candidate_result r;
    mtd::chain8_one<VIS>(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
    o.combo = c;
    o.cost = r.cost;
    o.distortion = r.distortion;
    o.bits = r.bits;
    o.satd = r.satd;
    o.eob = r.eob;
  }
  best[b] = o;
}

// Device address of g_noalloc_keys in the current device's context.  The
// symbol name is only a host-side handle; the address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every call
// (a table lookup once the module is loaded), so a context that was destroyed
// and created again (cudaDeviceReset) gets its own array's address.
int noalloc_keys_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_keys) != cudaSuccess || !p) return MT_ERR_DEVICE;
  *out = p;
  return MT_OK;
}

}  // namespace

extern "C" int mt_rdo_level8_device_noalloc(const uint16_t* d_src, const uint16_t* d_recon,
                                            const mt_chain_params* prm, const mt_quant* quant,
                                            const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                                            const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos,
                                            int32_t ncombos, mt_block_best* d_best, void* stream) {
  // The checks and codes of mt_rdo_level8_device, then this entry point's own
  // array bound.
  if (!prm || !quant) return MT_ERR_INVALID_INPUT;
  if (prm->tx_size != 8 || prm->bd != 8) return MT_ERR_UNSUPPORTED;
  if (prm->frame_w <= 0 || prm->frame_h <= 0 || prm->stride < prm->frame_w) return MT_ERR_INVALID_INPUT;
  if (nblocks < 0 || ncombos < 0) return MT_ERR_INVALID_INPUT;
  if (nblocks == 0 || ncombos == 0) return MT_OK;
  if ((long long)nblocks * ncombos > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  if (ncombos > MT_LEVEL_MAX_COMBOS) return MT_ERR_TOO_LARGE;
  if (nblocks > MT_NOALLOC_MAX_BLOCKS) return MT_ERR_TOO_LARGE;
  if (!d_src || !d_recon || !d_costs || !d_blocks || !d_combos || !d_best) return MT_ERR_INVALID_INPUT;
  void* keys_addr = nullptr;
  int rc = noalloc_keys_address(&keys_addr);
  if (rc != MT_OK) return rc;
  unsigned long long* keys = static_cast<unsigned long long*>(keys_addr);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  NoAllocArgs a;
  a.p = *prm;
  a.q = *quant;
  a.trellis_lambda = mth::scaled_trellis_lambda_host((float)quant->dc_q, prm->trellis_lambda0);
  a.has_qm = d_qm_row != nullptr;
  if (cudaMemsetAsync(keys, 0xff, (size_t)nblocks * sizeof(unsigned long long), st) != cudaSuccess)
    return MT_ERR_DEVICE;
  const long long total = (long long)nblocks * ncombos;
  const unsigned grid = (unsigned)((total + kNoAllocThreads - 1) / kNoAllocThreads);
  // A frame displayed smaller than coded masks the samples past its edge.
  const bool vis = (prm->vis_w > 0 && prm->vis_w < prm->frame_w) || (prm->vis_h > 0 && prm->vis_h < prm->frame_h);
  if (vis)
    noalloc_keys_kernel<true><<<grid, kNoAllocThreads, 0, st>>>(d_src, d_recon, a, d_qm_row, d_costs, d_blocks, nblocks,
                                                         d_combos, ncombos, keys);
  else
    noalloc_keys_kernel<false><<<grid, kNoAllocThreads, 0, st>>>(d_src, d_recon, a, d_qm_row, d_costs, d_blocks, nblocks,
                                                         d_combos, ncombos, keys);
  if (vis)
    noalloc_winner_kernel<true><<<(nblocks + kNoAllocThreads - 1) / kNoAllocThreads, kNoAllocThreads, 0, st>>>(
      d_src, d_recon, a, d_qm_row, d_costs, d_blocks, nblocks, d_combos, keys, d_best);
  else
    noalloc_winner_kernel<false><<<(nblocks + kNoAllocThreads - 1) / kNoAllocThreads, kNoAllocThreads, 0, st>>>(
      d_src, d_recon, a, d_qm_row, d_costs, d_blocks, nblocks, d_combos, keys, d_best);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}
