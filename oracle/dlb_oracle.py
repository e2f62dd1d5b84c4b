"""CPU restatement of the reference's load-balancing planner -- test
infrastructure only (tests/ and the golden-fixture script import it; the
product's planner is eu3d_dlb_plan in the CUDA library).

DynamicLoadBalancer::DLBPriorityQueue (src/LoadBalance.cpp:8-59):
  average = integer mean of the loads (Array::AveValue, include/Array.hpp:314-318);
  ranks with load >= average go into `maxHeap`, the others into `minHeap`,
  both std::priority_queue<std::pair<int, int>> of (load, rank) -- so both
  pop the LARGEST (load, rank) first;
  each sender popped from maxHeap passes min(excess, room) to receivers
  popped from minHeap until its excess (taken at push time) is gone; a
  receiver still below the average is pushed back with its new load.
"""
from __future__ import annotations

import heapq


def dlb_plan(loads):
    arr = [int(v) for v in loads]
    n = len(arr)
    if n == 0:
        return []
    average = sum(arr) // n  # C++ int division of non-negative sums
    over, under = [], []     # heapq is a min-heap: store negated pairs
    for i, v in enumerate(arr):
        heapq.heappush(over if v >= average else under, (-v, -i))
    out = []
    while over:
        v, i = heapq.heappop(over)
        sender, diff = -i, -v - average
        while under and diff > 0:
            w, r = heapq.heappop(under)
            receiver, surplus = -r, average - (-w)
            x = min(diff, surplus)
            arr[sender] -= x
            arr[receiver] += x
            out.append((sender, receiver, x))
            diff -= x
            if arr[receiver] < average:
                heapq.heappush(under, (-arr[receiver], -receiver))
    return out
