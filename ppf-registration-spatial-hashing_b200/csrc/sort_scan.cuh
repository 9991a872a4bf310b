// Device-wide primitives written for this engine: a stable LSD radix sort of
// (key, uint32 value) pairs and run-table construction over sorted keys.
#pragma once

#include "common.cuh"

namespace ppf {

// Stable LSD radix sort, 8-bit digits, one "onesweep" kernel per digit:
// each tile ranks its keys with warp multisplit, publishes per-digit counts
// and resolves its global offsets by decoupled look-back over the preceding
// tiles (tiles are numbered in launch order through an atomic counter, so
// every tile it waits on is already resident).  Waits are bounded; a wait
// that gives up raises kFlagSpinTimeout in *flags.
//
// keys/vals hold the input and receive the output (n elements each);
// vals == nullptr is not allowed, vals_iota makes the input values 0..n-1
// (vals is then output-only).  Digits [begin_bit, end_bit) are sorted; bits
// outside that range must not matter to the caller's order.  A sort whose
// look-back gave up leaves its output undefined (but every write inside the
// buffers): sort() waits for the stream, reads the flag and raises
// PPF_ERR_TIMEOUT, so nothing downstream reads that output.
template <typename K>
class RadixSorter {
 public:
  void sort(K* keys, uint32_t* vals, bool vals_iota, size_t n, int begin_bit, int end_bit,
            cudaStream_t st, uint32_t* d_flags);
  size_t launches() const { return launches_; }
  // Test hook: in the next sort of at least two tiles, tile 1 of the first
  // pass never publishes its look-back status and the waits on it are limited
  // to a few thousand spins.
  void arm_stall() { stall_ = true; }
  void release() {
    kalt_.release();
    valt_.release();
    hist_.release();
    status_.release();
    counters_.release();
  }

 private:
  DevBuf kalt_, valt_, hist_, status_, counters_;
  size_t launches_ = 0;
  bool stall_ = false;
};

extern template class RadixSorter<uint32_t>;
extern template class RadixSorter<unsigned long long>;

// Run table of a sorted key array: K unique keys, the first position of each
// run and its length.  Returns K (synchronises the stream once to read it).
// uniq/first/count must have room for n entries.
size_t build_runs(const uint32_t* sorted_keys, size_t n, uint32_t* uniq, uint32_t* first,
                  uint32_t* count, DevBuf& scratch, cudaStream_t st, size_t* launches);
// The same with outputs allocated at their final size K (no n-sized temporaries).
size_t build_runs(const uint32_t* sorted_keys, size_t n, DevBuf& uniq, DevBuf& first, DevBuf& count,
                  DevBuf& scratch, cudaStream_t st, size_t* launches);

// In-place exclusive scan of n uint32 by one block (for per-run tables of at
// most a few million entries); *total_dev receives the sum.
void exclusive_scan_small(uint32_t* v, size_t n, uint32_t* total_dev, cudaStream_t st);

}  // namespace ppf
