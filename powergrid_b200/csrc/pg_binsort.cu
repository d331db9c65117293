// Stable counting sort of samples by bin key on the device.
//
// The adjoint gridding processes samples bin by bin (bins = segment window x
// tile), in their original order inside a bin.  This is the same permutation
// a stable CPU counting sort (or numpy's stable argsort) produces, so it is
// bit-exact against one:
//   1. count:   every block counts the keys of one contiguous chunk of the
//               input into counts[key][block] (key-major);
//   2. scan:    an exclusive scan of counts in key-major order gives, for
//               every (key, block), the first output slot of that block's
//               elements with that key (blocks in input order inside a key);
//   3. scatter: one warp per chunk walks it in input order, 32 elements at a
//               time; lanes with equal keys (__match_any_sync) take
//               consecutive slots in lane order from the (key, block)
//               cursor.
// Every step is deterministic; the order within a bin is the input order.
#include <algorithm>

#include "pg_binsort.cuh"

namespace pg {
namespace {

constexpr int kScanThreads = 256;

__global__ void k_bin_count(const uint32_t* __restrict__ key, uint64_t M, uint64_t chunk, int nblk,
                            uint32_t* __restrict__ counts) {
  const uint64_t b = blockIdx.x;
  const uint64_t lo = b * chunk, hi = min(M, lo + chunk);
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&counts[(uint64_t)key[i] * nblk + b], 1u);
}

// Exclusive scan in three passes over segments of `seg` elements.
__global__ void k_scan_sums(const uint32_t* __restrict__ v, uint64_t n, uint64_t seg, uint64_t* __restrict__ sums) {
  __shared__ uint64_t red[kScanThreads];
  const uint64_t lo = (uint64_t)blockIdx.x * seg, hi = min(n, lo + seg);
  uint64_t a = 0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) a += v[i];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int o = kScanThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = red[0];
}

__global__ void k_scan_block_sums(uint64_t* __restrict__ sums, int nseg) {
  if (threadIdx.x != 0) return;
  uint64_t run = 0;
  for (int i = 0; i < nseg; ++i) { const uint64_t t = sums[i]; sums[i] = run; run += t; }
}

// Each thread takes a contiguous piece of the block's segment: piece sums,
// a block exclusive scan of them, then the piece is rewritten exclusively.
__global__ void k_scan_apply(uint32_t* __restrict__ v, uint64_t n, uint64_t seg, const uint64_t* __restrict__ sums) {
  __shared__ uint64_t part[kScanThreads];
  const uint64_t lo = (uint64_t)blockIdx.x * seg, hi = min(n, lo + seg);
  const uint64_t per = (seg + kScanThreads - 1) / kScanThreads;
  const uint64_t a = min(hi, lo + threadIdx.x * per), e = min(hi, a + per);
  uint64_t s = 0;
  for (uint64_t i = a; i < e; ++i) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t run = sums[blockIdx.x];
    for (int t = 0; t < kScanThreads; ++t) { const uint64_t x = part[t]; part[t] = run; run += x; }
  }
  __syncthreads();
  uint64_t run = part[threadIdx.x];
  for (uint64_t i = a; i < e; ++i) { const uint32_t x = v[i]; v[i] = (uint32_t)run; run += x; }
}

__global__ void k_bin_starts(const uint32_t* __restrict__ cursor, uint64_t nkeys, int nblk,
                             uint32_t* __restrict__ starts) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nkeys) starts[k] = cursor[k * nblk];
}

__global__ void k_bin_scatter(const uint32_t* __restrict__ key, uint64_t M, uint64_t chunk, int nblk,
                              uint32_t* __restrict__ cursor, uint32_t* __restrict__ perm) {
  const uint64_t b = blockIdx.x;
  const uint64_t lo = b * chunk, hi = min(M, lo + chunk);
  const int lane = threadIdx.x;
  const unsigned lt = (1u << lane) - 1u;
  for (uint64_t base = lo; base < hi; base += 32) {
    const uint64_t i = base + lane;
    const bool live = i < hi;
    const uint32_t k = live ? key[i] : 0xffffffffu;
    const unsigned same = __match_any_sync(0xffffffffu, k);
    const int leader = __ffs(same) - 1;
    uint32_t slot = 0;
    if (live && lane == leader) {
      uint32_t* c = &cursor[(uint64_t)k * nblk + b];
      slot = *c;
      *c = slot + __popc(same);
    }
    slot = __shfl_sync(0xffffffffu, slot, leader);
    if (live) perm[slot + __popc(same & lt)] = (uint32_t)i;
  }
}

}  // namespace

pg_status bin_sort(const uint32_t* key, uint64_t M, uint64_t nkeys, uint32_t* perm, uint32_t* starts,
                   cudaStream_t s) {
  if (M == 0) return PG_OK;
  if (M >= (1ull << 32)) return set_error(PG_INVALID_ARG, "bin sort: too many samples");
  // chunks of >= 1024 samples; the (key, chunk) table stays below 16 M entries
  uint64_t nblk = (M + 1023) / 1024;
  const uint64_t cap = 16ull << 20;
  if (nblk * nkeys > cap) nblk = std::max<uint64_t>(1, cap / std::max<uint64_t>(1, nkeys));
  nblk = std::min<uint64_t>(nblk, 65535);
  const uint64_t chunk = (M + nblk - 1) / nblk;
  nblk = (M + chunk - 1) / chunk;
  const uint64_t n = nkeys * nblk;
  DevBuf<uint32_t> table;
  PG_TRY(table.alloc(n));
  PG_CUDA(cudaMemsetAsync(table.p, 0, n * sizeof(uint32_t), s));
  PG_LAUNCH(k_bin_count, (unsigned)nblk, 256, 0, s, key, M, chunk, (int)nblk, table.p);
  const uint64_t seg = 8192;
  const uint64_t nseg = (n + seg - 1) / seg;
  DevBuf<uint64_t> sums;
  PG_TRY(sums.alloc(nseg));
  PG_LAUNCH(k_scan_sums, (unsigned)nseg, kScanThreads, 0, s, table.p, n, seg, sums.p);
  PG_LAUNCH(k_scan_block_sums, 1, 32, 0, s, sums.p, (int)nseg);
  PG_LAUNCH(k_scan_apply, (unsigned)nseg, kScanThreads, 0, s, table.p, n, seg, sums.p);
  PG_LAUNCH(k_bin_starts, ceil_div(nkeys, 256), 256, 0, s, table.p, nkeys, (int)nblk, starts);
  PG_LAUNCH(k_bin_scatter, (unsigned)nblk, 32, 0, s, key, M, chunk, (int)nblk, table.p, perm);
  // table and sums are released on return: wait for the kernels that use them
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

}  // namespace pg
