// Stable device counting sort of samples by bin key (pg_binsort.cu).
#pragma once

#include "pg_common.cuh"

namespace pg {

// perm[j] = index of the j-th sample in (key, input index) order; starts[k] =
// first sorted position of key k (nkeys entries).  key < nkeys.
pg_status bin_sort(const uint32_t* key, uint64_t M, uint64_t nkeys, uint32_t* perm, uint32_t* starts,
                   cudaStream_t s);

}  // namespace pg
