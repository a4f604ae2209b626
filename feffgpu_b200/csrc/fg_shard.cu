// fg_shard.cu -- the multi-GPU split of a path list (host code): longest-processing-time-first assignment.
#include <algorithm>
#include <functional>
#include <numeric>
#include <queue>
#include <string>
#include <utility>
#include <vector>

#include "feffgpu_b200.h"
#include "fg_launch.h"

// Paths in order of decreasing cost (equal costs in index order) each go to the least-loaded rank (equal loads: the
// lowest rank), with a binary heap of the ranks' loads: O(n log n + n log world).
extern "C" fg_status fg_shard_lpt(const double *cost, int64_t n, int32_t world, int32_t *owner)
{
    if (n < 0 || world < 1) return fg::fail(FG_ERR_VALUE, "n must be >= 0 and world >= 1");
    if (n > 0 && (!cost || !owner)) return fg::fail(FG_ERR_VALUE, "null array");
    std::vector<int64_t> order((size_t)n);
    std::iota(order.begin(), order.end(), int64_t(0));
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    using Load = std::pair<double, int32_t>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int32_t r = 0; r < world; ++r) heap.push({0.0, r});
    for (int64_t i : order) {
        const Load top = heap.top();
        heap.pop();
        owner[i] = top.second;
        heap.push({top.first + cost[i], top.second});
    }
    return FG_OK;
}
