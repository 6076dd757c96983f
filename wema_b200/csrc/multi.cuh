// multi.cuh - one launch over many video streams.
//
// A batched launch concatenates the grids of its tasks (one task = one
// stream's launch of that kernel).  The task map, in device memory, is
//   map[0] = n,  map[1 .. n+1] = first block of each task (map[n+1] = total),
//   map[n+2 .. 2n+1] = grid x of each task,  map[2n+2 .. 3n+1] = grid y,
// and a block finds its task by binary search, then its local (x, y, z).
#pragma once

namespace wema {

struct TaskBlock {
    int task, x, y, z;
};

__device__ __forceinline__ TaskBlock task_block(const int* map, int b) {
    const int n = map[0];
    const int* start = map + 1;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    TaskBlock t;
    t.task = lo;
    int r = b - start[lo];
    const int gx = map[n + 2 + lo], gy = map[2 * n + 2 + lo];
    t.x = r % gx;
    r /= gx;
    t.y = r % gy;
    t.z = r / gy;
    return t;
}

}  // namespace wema
