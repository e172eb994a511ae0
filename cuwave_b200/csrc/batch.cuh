// A batch of 2D problems stepped together: many shots, and many grids of uneven size and
// order, one launch a step per stencil radius.
//
// Each item is one problem's step: its own geometry, stencil row, factors, material,
// levels, folded sources and refill (a StepParams and a Fold2, the quad step's). Items of
// one radius share a launch: the launch's threads are the items' units (quads x row
// chunks) laid end to end, each item padded to whole blocks so that a block steps one
// item, and a thread finds its item by bisection over the items' first threads. An item
// rests from its own step count on, so problems of different lengths march together.
// The receivers of every item are read after the step by one launch over all of them.
#pragma once

#include "step2d.cuh"

namespace cwb {

template <typename T>
struct Batch2Item {
  StepParams<T> s;
  Fold2<T> fold;
  long long first;  // the item's first thread in its launch
  int steps;        // the item rests from t = steps on
};

template <typename T>
struct Batch2Params {
  const Batch2Item<T> *items;
  int count;
  long long total;  // threads of the launch
  int flags;        // K_ADV
  int hold;         // an item has a Dirichlet face
  int pml;          // an item has a pml
  int *ctr;
};

// HOLD: an item of the launch has a Dirichlet face (without one, the wall tests fold away);
// PML: an item has a pml (without one, the step carries no slab code)
template <typename T, int R, bool HOLD = true, bool PML = true>
__global__ void __launch_bounds__(S2_THREADS, Step2Shape<T, R>::MIN_BLOCKS)
    batch2d_kernel(const __grid_constant__ Batch2Params<T> p) {
  static_assert(Step2Shape<T, R>::SUPPORTED, "the 2D quad step is built for float");
  const int t = step_index(p.ctr);
  const long long k = (long long)blockIdx.x * S2_THREADS + threadIdx.x;
  if (k < p.total) {
    int lo = 0, hi = p.count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.items[mid].first <= k)
        lo = mid;
      else
        hi = mid - 1;
    }
    const Batch2Item<T> &it = p.items[lo];
    if (t < it.steps)
      step2d_rows<T, R, HOLD, PML>(it.s, t, k - it.first, it.fold);
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

// the receivers of every item: sensor j of the batch is column col[j] of item owner[j]'s
// record, row t, read from the item's level after its step
template <typename T>
struct BatchRecord {
  DLevel a;
  const int *lin;
  T *record;  // (steps, num)
  int num;
  int steps;
};

template <typename T>
struct BatchRecordParams {
  const BatchRecord<T> *recs;
  const int *owner;
  const int *col;
  int total;
  int flags;
  int *ctr;
};

template <typename T>
__global__ void batch_record_kernel(const __grid_constant__ BatchRecordParams<T> p) {
  const int t = step_index(p.ctr);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.total) {
    const BatchRecord<T> &r = p.recs[p.owner[j]];
    if (t < r.steps) {
      const int c = p.col[j];
      r.record[(long long)t * r.num + c] = level<T>(r.a, t)[r.lin[c]];
    }
  }
  finish_step(p.ctr, p.flags & K_ADV);
}

}  // namespace cwb
