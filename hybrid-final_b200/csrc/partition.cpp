// partition.cpp -- cases -> devices for the batched and served forms on the
// GPUs of one node.
//
// Independent cases have no exchange step, so a set of them shards by case:
// each device runs its own share as one batch and the host gathers the
// per-case results.  The placement is longest-first greedy: cases in
// decreasing weight (ties: lower case index first) each go to the device
// with the least weight placed so far among the devices whose byte budget
// still holds the case (ties: lower device index).  It depends only on its
// inputs, so every rank of a job computes the same placement without
// exchanging it.
#include <algorithm>
#include <numeric>
#include <vector>

#include "capi_internal.hpp"

extern "C" hp_status hp_partition_cases(const double *weight, const size_t *bytes, int ncases, int ndevices,
                                        const size_t *budget, int *device_of) {
    using hpi::set_error;
    if (ncases < 0 || ndevices <= 0 || (ncases > 0 && (!weight || !bytes || !device_of)))
        return set_error("hp_partition_cases: bad arguments"), HP_ERR_ARG;
    for (int k = 0; k < ncases; k++)
        if (!(weight[k] >= 0.0)) return set_error("hp_partition_cases: weights must be finite and >= 0"), HP_ERR_ARG;
    std::vector<int> order(ncases);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return weight[a] > weight[b]; });
    std::vector<double> load(ndevices, 0.0);
    std::vector<size_t> used(ndevices, 0);
    hp_status st = HP_OK;
    for (int k : order) {
        int best = -1;
        for (int g = 0; g < ndevices; g++) {
            if (budget && (bytes[k] > budget[g] || used[g] > budget[g] - bytes[k])) continue;
            if (best < 0 || load[g] < load[best]) best = g;
        }
        device_of[k] = best;
        if (best < 0) {
            if (st == HP_OK) set_error("hp_partition_cases: a case is larger than every device's remaining budget");
            st = HP_ERR_CAPACITY;
            continue;
        }
        load[best] += weight[k];
        used[best] += bytes[k];
    }
    return st;
}
