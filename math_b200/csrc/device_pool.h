// Device memory for the library's buffers, cached for reuse.
//
// Every scene and painter allocates its device buffers through this pool.
// A released buffer is kept, by device and rounded size, and handed to the
// next request of that size instead of returning it to the driver, so jobs
// that follow one another (a serving loop, a benchmark) neither pay for
// cudaMalloc nor for cudaFree, which synchronizes the whole device.  Sizes
// are rounded to a power of two up to 1 MiB and to a multiple of 2 MiB above.
//
// A buffer is released only by its owner after the owner's work on it has
// finished (painters synchronize their stream before releasing, scenes are
// released after their painters), so reuse needs no further ordering.
// When the device is out of memory the cached buffers are freed and the
// allocation retried.
#pragma once

#include <cstddef>

namespace nbpt::pool
{
void* allocate(std::size_t bytes, int* device);
void release(void* p, std::size_t bytes, int device);
// frees every cached buffer of every device; returns the bytes freed
std::size_t trim();
// bytes held in the cache
std::size_t cached();
} // namespace nbpt::pool
