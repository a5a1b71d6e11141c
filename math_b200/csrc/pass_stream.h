// Passes of a painter on a worker thread, each pass's images handed to a
// callback: the reference painter's thread and Notifier
// (src/painter/painter.cpp:77-134, painter.h:36-78) for callers of the C ABI.
#pragma once

#include "painter_api.h"

#include <atomic>
#include <mutex>
#include <string>
#include <thread>

namespace nbpt
{
// Two pinned host image buffers and an event for each: pinning host memory
// is slow, so a painter keeps its buffers from one start to the next.
class PassBuffers final
{
public:
        explicit PassBuffers(long long pixel_count);
        ~PassBuffers();

        PassBuffers(const PassBuffers&) = delete;
        PassBuffers& operator=(const PassBuffers&) = delete;

        long long pixel_count;
        float* rgb[2] = {nullptr, nullptr};
        float* rgba[2] = {nullptr, nullptr};
        void* done[2] = {nullptr, nullptr}; // cudaEvent_t

private:
        void release();
};

class PassStream final
{
public:
        using PassCallback = void (*)(void* user, long long pass, const float* rgb, const float* rgba,
                                      long long pixel_count);
        using ErrorCallback = void (*)(void* user, const char* message);

        // Runs `max_passes` passes (0: until stop()).  While pass k + 1 renders,
        // the images of pass k go to `on_pass` on the worker thread.
        PassStream(Painter* painter, PassBuffers* buffers, int max_passes, PassCallback on_pass,
                   ErrorCallback on_error, void* user);
        ~PassStream();

        PassStream(const PassStream&) = delete;
        PassStream& operator=(const PassStream&) = delete;

        // asks the worker to stop after the pass in flight and waits for it
        void stop();
        // asks the worker to stop after the pass in flight, without waiting
        void request_stop();
        // waits for the worker to end
        void join();
        bool running() const;
        long long passes() const;

private:
        void run();

        Painter* painter_;
        PassBuffers* buffers_;
        int max_passes_;
        PassCallback on_pass_;
        ErrorCallback on_error_;
        void* user_;
        std::atomic<bool> stop_{false};
        std::atomic<bool> running_{true};
        std::atomic<long long> passes_{0};
        std::mutex join_mutex_;
        std::thread worker_;
};
} // namespace nbpt
