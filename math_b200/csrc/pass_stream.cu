// Passes of a painter on a worker thread (pass_stream.h).
#include "pass_stream.h"

#include "cuda_error.h"

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
                throw CudaError(what, e);
        }
}

} // namespace

PassBuffers::PassBuffers(const long long pixels)
        : pixel_count(pixels)
{
        try
        {
                for (int i = 0; i < 2; ++i)
                {
                        check(cudaHostAlloc(reinterpret_cast<void**>(&rgb[i]), pixels * 3 * sizeof(float),
                                            cudaHostAllocDefault),
                              "cudaHostAlloc");
                        check(cudaHostAlloc(reinterpret_cast<void**>(&rgba[i]), pixels * 4 * sizeof(float),
                                            cudaHostAllocDefault),
                              "cudaHostAlloc");
                        cudaEvent_t e = nullptr;
                        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
                        done[i] = e;
                }
        }
        catch (...)
        {
                release();
                throw;
        }
}

PassBuffers::~PassBuffers()
{
        release();
}

void PassBuffers::release()
{
        for (int i = 0; i < 2; ++i)
        {
                if (done[i])
                {
                        cudaEventSynchronize(static_cast<cudaEvent_t>(done[i]));
                        cudaEventDestroy(static_cast<cudaEvent_t>(done[i]));
                        done[i] = nullptr;
                }
                if (rgb[i])
                {
                        cudaFreeHost(rgb[i]);
                        rgb[i] = nullptr;
                }
                if (rgba[i])
                {
                        cudaFreeHost(rgba[i]);
                        rgba[i] = nullptr;
                }
        }
}

PassStream::PassStream(
        Painter* const painter,
        PassBuffers* const buffers,
        const int max_passes,
        const PassCallback on_pass,
        const ErrorCallback on_error,
        void* const user)
        : painter_(painter),
          buffers_(buffers),
          max_passes_(max_passes),
          on_pass_(on_pass),
          on_error_(on_error),
          user_(user)
{
        if (!painter || !buffers || !on_pass)
        {
                throw std::runtime_error("a pass stream needs a painter, its buffers and a pass callback");
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

void PassStream::request_stop()
{
        stop_ = true;
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
                PassBuffers& b = *buffers_;
                const auto stream = static_cast<cudaStream_t>(painter_->stream());
                const auto launch = [&](const int slot)
                {
                        painter_->enqueue_passes(1);
                        painter_->enqueue_images(b.rgb[slot], b.rgba[slot]);
                        check(cudaEventRecord(static_cast<cudaEvent_t>(b.done[slot]), stream), "cudaEventRecord");
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
                        check(cudaEventSynchronize(static_cast<cudaEvent_t>(b.done[slot])), "pass");
                        passes_ = k + 1;
                        on_pass_(user_, k + 1, b.rgb[slot], b.rgba[slot], b.pixel_count);
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
