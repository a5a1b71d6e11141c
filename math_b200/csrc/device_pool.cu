// Device memory cache of the library's buffers (device_pool.h).
#include "device_pool.h"

#include "cuda_error.h"

#include <cuda_runtime.h>

#include <iterator>
#include <map>
#include <unordered_map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace nbpt::pool
{
namespace
{
struct Cache final
{
        std::mutex mutex;
        // device -> (rounded size -> free buffers)
        std::map<int, std::multimap<std::size_t, void*>> free;
        // buffers handed out for a smaller request than their size
        std::unordered_map<void*, std::size_t> larger;
        std::size_t bytes = 0;
};

Cache& cache()
{
        static Cache* const c = new Cache; // lives for the process: buffers may be released at exit
        return *c;
}

std::size_t rounded(const std::size_t bytes)
{
        constexpr std::size_t SMALL = std::size_t{1} << 20;
        constexpr std::size_t LARGE_STEP = std::size_t{2} << 20;
        if (bytes <= SMALL)
        {
                std::size_t r = 256;
                while (r < bytes)
                {
                        r <<= 1;
                }
                return r;
        }
        return (bytes + LARGE_STEP - 1) / LARGE_STEP * LARGE_STEP;
}

std::size_t free_device(std::multimap<std::size_t, void*>& blocks)
{
        std::size_t n = 0;
        for (const auto& [size, p] : blocks)
        {
                cudaFree(p);
                n += size;
        }
        blocks.clear();
        return n;
}
} // namespace

void* allocate(const std::size_t bytes, int* const device)
{
        int d = 0;
        cudaError_t e = cudaGetDevice(&d);
        if (e != cudaSuccess)
        {
                throw CudaError("cudaGetDevice", e);
        }
        *device = d;
        const std::size_t size = rounded(bytes);
        Cache& c = cache();
        {
                const std::lock_guard lock(c.mutex);
                auto& blocks = c.free[d];
                // small sizes: the same power of two; large ones: the smallest
                // cached buffer that holds the request with at most a quarter
                // to spare (jobs of similar sizes reuse one another's buffers)
                const auto i = blocks.lower_bound(size);
                if (i != blocks.end() && (i->first == size || (size > (std::size_t{1} << 20) &&
                                                               i->first <= size + size / 4)))
                {
                        void* const p = i->second;
                        const std::size_t have = i->first;
                        blocks.erase(i);
                        c.bytes -= have;
                        if (have != size)
                        {
                                c.larger[p] = have;
                        }
                        return p;
                }
        }
        void* p = nullptr;
        e = cudaMalloc(&p, size);
        while (e == cudaErrorMemoryAllocation)
        {
                // give cached buffers back to the driver, the largest first,
                // until the request fits (each cudaFree waits for the device)
                cudaGetLastError();
                {
                        const std::lock_guard lock(c.mutex);
                        auto& blocks = c.free[d];
                        if (blocks.empty())
                        {
                                break;
                        }
                        const auto last = std::prev(blocks.end());
                        cudaFree(last->second);
                        c.bytes -= last->first;
                        blocks.erase(last);
                }
                e = cudaMalloc(&p, size);
        }
        if (e != cudaSuccess)
        {
                cudaGetLastError();
                throw CudaError("cudaMalloc of " + std::to_string(size) + " bytes", e);
        }
        return p;
}

void release(void* const p, const std::size_t bytes, const int device)
{
        if (!p)
        {
                return;
        }
        Cache& c = cache();
        const std::lock_guard lock(c.mutex);
        std::size_t size = rounded(bytes);
        const auto l = c.larger.find(p);
        if (l != c.larger.end())
        {
                size = l->second;
                c.larger.erase(l);
        }
        c.free[device].emplace(size, p);
        c.bytes += size;
}

std::size_t trim()
{
        Cache& c = cache();
        const std::lock_guard lock(c.mutex);
        std::size_t n = 0;
        int current = 0;
        const bool has_current = cudaGetDevice(&current) == cudaSuccess;
        for (auto& [device, blocks] : c.free)
        {
                if (blocks.empty())
                {
                        continue;
                }
                cudaSetDevice(device);
                n += free_device(blocks);
        }
        if (has_current)
        {
                cudaSetDevice(current);
        }
        cudaGetLastError();
        c.bytes -= n;
        return n;
}

std::size_t cached()
{
        Cache& c = cache();
        const std::lock_guard lock(c.mutex);
        return c.bytes;
}
} // namespace nbpt::pool
