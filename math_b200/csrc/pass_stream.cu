// Passes of a painter on a worker thread (pass_stream.h).
#include "pass_stream.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace nbpt
{
namespace
{
void check(const cudaError_t e, const char* what)
{
        if (e != cudaSuccess)
        {
                throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
        }
}

// two pinned image buffers and an event for each
struct Slots final
{
        float* rgb[2] = {nullptr, nullptr};
        float* rgba[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};

        explicit Slots(const long long pixels)
        {
                for (int i = 0; i < 2; ++i)
                {
                        check(cudaHostAlloc(reinterpret_cast<void**>(&rgb[i]), pixels * 3 * sizeof(float),
                                            cudaHostAllocDefault),
                              "cudaHostAlloc");
                        check(cudaHostAlloc(reinterpret_cast<void**>(&rgba[i]), pixels * 4 * sizeof(float),
                                            cudaHostAllocDefault),
                              "cudaHostAlloc");
                        check(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
                }
        }

        ~Slots()
        {
                for (int i = 0; i < 2; ++i)
                {
                        if (done[i])
                        {
                                cudaEventSynchronize(done[i]);
                                cudaEventDestroy(done[i]);
                        }
                        cudaFreeHost(rgb[i]);
                        cudaFreeHost(rgba[i]);
                }
        }

        Slots(const Slots&) = delete;
        Slots& operator=(const Slots&) = delete;
};
} // namespace

PassStream::PassStream(
        Painter* const painter,
        const long long pixel_count,
        const int max_passes,
        const PassCallback on_pass,
        const ErrorCallback on_error,
        void* const user)
        : painter_(painter),
          pixel_count_(pixel_count),
          max_passes_(max_passes),
          on_pass_(on_pass),
          on_error_(on_error),
          user_(user)
{
        if (!painter || !on_pass)
        {
                throw std::runtime_error("a pass stream needs a painter and a pass callback");
        }
        if (max_passes < 0)
        {
                throw std::runtime_error("pass count must not be negative");
        }
        worker_ = std::thread(&PassStream::run, this);
}

PassStream::~PassStream()
{
        stop();
}

void PassStream::stop()
{
        stop_ = true;
        join();
}

void PassStream::join()
{
        const std::lock_guard lock(join_mutex_);
        if (worker_.joinable() && worker_.get_id() != std::this_thread::get_id())
        {
                worker_.join();
        }
}

bool PassStream::running() const
{
        return running_;
}

long long PassStream::passes() const
{
        return passes_;
}

void PassStream::run()
{
        try
        {
                check(cudaSetDevice(painter_->device()), "cudaSetDevice");
                const Slots slots(pixel_count_);
                const auto stream = static_cast<cudaStream_t>(painter_->stream());
                const auto launch = [&](const int slot)
                {
                        painter_->enqueue_passes(1);
                        painter_->enqueue_images(slots.rgb[slot], slots.rgba[slot]);
                        check(cudaEventRecord(slots.done[slot], stream), "cudaEventRecord");
                };
                launch(0);
                for (long long k = 0;; ++k)
                {
                        const int slot = static_cast<int>(k & 1);
                        const bool more = !stop_ && (max_passes_ == 0 || k + 1 < max_passes_);
                        if (more)
                        {
                                launch(1 - slot);
                        }
                        check(cudaEventSynchronize(slots.done[slot]), "pass");
                        passes_ = k + 1;
                        on_pass_(user_, k + 1, slots.rgb[slot], slots.rgba[slot], pixel_count_);
                        if (!more)
                        {
                                break;
                        }
                }
                painter_->wait(); // statistics of the last pass
        }
        catch (const std::exception& e)
        {
                cudaGetLastError();
                if (on_error_)
                {
                        on_error_(user_, e.what());
                }
        }
        running_ = false;
}
} // namespace nbpt
