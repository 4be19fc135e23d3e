// Slot layout and probing shared by the key table and its device-side users.
#pragma once
#include "ngs_common.cuh"

static constexpr unsigned long long kEmpty = 0xFFFFFFFFFFFFFFFFull;

struct __align__(16) Slot {
  unsigned long long key;
  long long val;
};

NGS_DEV unsigned long long mix64(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

// Device-side lookup used by the dual-grid accumulation through a key table.
NGS_DEV long long table_find_single(const Slot* __restrict__ slots, int64_t mask, unsigned long long key) {
  int64_t slot = (int64_t)(mix64(key) & (unsigned long long)mask);
  for (int64_t probe = 0; probe <= mask; probe++) {
    const Slot v = slots[slot];
    if (v.key == key) return v.val;
    if (v.key == kEmpty) return -1;
    slot = (slot + 1) & mask;
  }
  return -1;
}
