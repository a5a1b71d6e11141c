// Render-job server: continuous batching of painters on one GPU.
//
// The reference renders one scene per painter, each painter with its own
// worker threads (src/painter/painter.cpp:77-134).  On one GPU many small
// renders would each leave most of the device idle, so the server runs many
// painters' passes at once: every admitted job has its own CUDA stream (the
// painter's), the server keeps one pass of every admitted job in flight, and
// jobs that arrive while others run are admitted as soon as a slot and
// device memory free up.  A job's result does not depend on what runs beside
// it: every path's random stream is fixed by (seed, pass, pixel, sample).
#pragma once

#include "painter_api.h"

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

namespace nbpt
{
enum class JobState : int
{
        QUEUED = 0,
        RUNNING = 1,
        DONE = 2,
        FAILED = 3
};

struct JobInfo final
{
        JobState state;
        int passes;
        int passes_done;
        long long footprint; // device bytes counted against the budget
        double submitted;    // seconds since the server started
        double started;      // admitted (-1 while queued)
        double finished;     // done or failed (-1 before)
        // device clock of the job's first pass start and last pass end, in
        // seconds after the server's reference event (-1 before the job is
        // done): CUDA events on the job's stream
        double device_started = -1;
        double device_finished = -1;
        std::string error;
};

class Server final
{
public:
        // max_jobs: jobs admitted at once; memory_budget: device bytes the
        // admitted jobs may hold (a job larger than the budget runs alone)
        Server(int max_jobs, long long memory_budget);
        ~Server();
        Server(const Server&) = delete;
        Server& operator=(const Server&) = delete;

        // The painter (and its scene) must stay alive and untouched by the
        // caller until the job is done or failed.
        long long submit(Painter* painter, int passes);
        // A render the server creates when it admits the job (so a queued job
        // holds no device memory) and owns until release(); the scene must
        // stay alive until then.
        long long submit_render(Scene* scene, int spp, int max_depth, std::uint32_t seed, int passes);
        // the images and statistics of a done job
        void images(long long job, float* rgb, float* rgba);
        Statistics statistics(long long job);
        // forgets a finished job and frees the painter the server created
        void release(long long job);
        JobInfo info(long long job) const;
        JobInfo wait(long long job);
        // A queued job fails at once with the error "cancelled"; a running
        // one stops taking paths in its pass in flight (Painter::cancel),
        // then fails the same way.  A finished job is left as it is.
        void cancel(long long job);
        // test hook: the next `count` renders the server creates fail as if
        // cudaMalloc had run out of device memory
        void fail_next_creations(int count);
        // test hook: while held, the server admits no job
        void hold_admission(bool hold);
        // device bytes of chunk buffers (the per-chunk path buffers of the
        // BPT kernels) of each render the server creates from now on; 0: an
        // equal share of the memory budget per slot, at least 4 GiB.  Larger
        // chunks leave less of each pass to the persistent kernels' tails;
        // fewer renders then fit in the budget at once.
        void set_chunk_budget(long long bytes);
        long long chunk_budget() const;
        double now() const;
        // finishes the running jobs, fails the queued ones and stops the
        // worker; the destructor calls it, and so does process exit for a
        // server never destroyed (before the CUDA runtime shuts down)
        void shutdown();

private:
        struct Job;
        std::shared_ptr<Job> find_locked(long long job) const;

        void run();
        bool admit_locked();
        long long slot_chunk_budget() const;
        void finish_locked(Job& job, JobState state, const std::string& error);

        int max_jobs_;
        long long budget_;
        long long initial_budget_ = 0;
        long long used_ = 0;
        double start_;
        mutable std::mutex mutex_;
        std::condition_variable changed_;
        std::map<long long, std::shared_ptr<Job>> jobs_;
        std::deque<std::shared_ptr<Job>> queue_;
        std::deque<std::shared_ptr<Job>> running_;
        long long next_id_ = 0;
        bool stop_ = false;
        int fail_creations_ = 0;
        bool hold_ = false;
        long long chunk_budget_ = 0; // set_chunk_budget
        void* reference_event_ = nullptr; // cudaEvent_t recorded at construction
        std::thread worker_;
};
} // namespace nbpt
