/*
 * faults.cpp - allocation-failure injection for tests (no counterpart in the
 * reference, whose loaders report failures through their status argument,
 * src/RTMCphon.f90:293-419).
 *
 * ptg_debug_fail_allocations(n) lets the next n allocations of the library
 * succeed and makes every later one fail (device buffers: cudaMalloc is not
 * called and the call returns PTG_ERR_NOMEM; host objects and arrays: the
 * allocation reports failure or throws std::bad_alloc, which the entry
 * points turn into PTG_ERR_NOMEM), until n < 0 turns injection off.  The
 * failures are made on the host; no device operation fails.
 */
#include <stdint.h>

#include <atomic>

#include "ptg_internal.h"

namespace ptg {

namespace {
std::atomic<int64_t> g_alloc_budget{-1};
}

bool alloc_should_fail() {
  int64_t b = g_alloc_budget.load(std::memory_order_relaxed);
  while (b >= 0) {
    if (b == 0) return true;
    if (g_alloc_budget.compare_exchange_weak(b, b - 1, std::memory_order_relaxed)) return false;
  }
  return false;
}

void alloc_check() {
  if (alloc_should_fail()) throw std::bad_alloc();
}

}  // namespace ptg

extern "C" int ptg_debug_fail_allocations(int64_t after) {
  ptg::g_alloc_budget.store(after < 0 ? -1 : after);
  return PTG_OK;
}
