// Item-list bookkeeping of the tensor-core sequence: closes a tensor-core
// product's item list (adds it to the statistics, resets the counters for
// the next product).
#include "launch.h"

namespace cfpq {
namespace {

__global__ void k_reset_list(IterState *st, int list) {
    st->items_total += st->item_count[list];
    st->items_by_variant[4] += st->item_count[list];
    st->item_count[list] = 0;
    st->item_next[list] = 0;
}

}  // namespace

cudaError_t launch_reset_list(IterState *st, int list, cudaStream_t s) {
    k_reset_list<<<1, 1, 0, s>>>(st, list);
    return cudaGetLastError();
}

}  // namespace cfpq
