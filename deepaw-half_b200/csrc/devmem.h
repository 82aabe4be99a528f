// Caching device allocator behind DeviceBuffer.
//
// cudaMalloc/cudaFree synchronise the device and can stall the calling host
// thread for tens to hundreds of milliseconds, which in a solve loop shows up
// as idle GPU time.  Freed blocks are therefore kept and reused:
//   * per host thread: a block freed by a thread is reused only by that
//     thread.  Every thread of the library issues its device work on one
//     stream (its Runtime's), so a reused block is stream-ordered after the
//     work that last touched it;
//   * when a thread ends, its blocks move to a process-wide pool after a
//     device synchronisation (all their work has finished), where any thread
//     may take them;
//   * a request takes the smallest cached block of at least its (rounded)
//     size and at most twice it; on an allocation failure every cached block
//     is released and the allocation retried once.
#pragma once

#include <cstddef>

namespace hb {

void* device_alloc(size_t bytes, size_t* granted);   // throws hb::Error on failure
void device_free(void* p, size_t granted);
void device_cache_release();                          // return cached blocks to the driver
// Process-wide counts since start: device_alloc calls (cached or not) and the
// cudaMalloc calls among them.
void device_alloc_counts(long long* requests, long long* driver_allocations);

}  // namespace hb
