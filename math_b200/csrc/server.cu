// Render-job server (server.h).
#include "server.h"

#include "cuda_error.h"


#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <set>
#include <vector>
#include <stdexcept>

namespace nbpt
{
namespace
{
double steady_seconds()
{
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Servers alive in the process: stopped at exit, before the CUDA runtime
// tears down, so that no worker thread is left issuing CUDA calls.
std::mutex g_live_mutex;
std::set<Server*>* g_live = nullptr;

void stop_live_servers()
{
        std::vector<Server*> live;
        {
                const std::lock_guard lock(g_live_mutex);
                if (g_live)
                {
                        live.assign(g_live->begin(), g_live->end());
                }
        }
        for (Server* s : live)
        {
                s->shutdown();
        }
}
} // namespace

struct Server::Job final
{
        long long id;
        Painter* painter = nullptr;
        // a render the server creates at admission
        Scene* scene = nullptr;
        int spp = 0;
        int max_depth = 0;
        std::uint32_t seed = 0;
        long long chunk_budget = 0; // the server's chunk budget when the render was submitted
        std::unique_ptr<Painter> owned;
        int device;
        JobInfo info;
        cudaEvent_t first = nullptr; // marks the start of the first pass
        cudaEvent_t done = nullptr;  // marks the end of the pass in flight
        bool pass_in_flight = false;
        std::atomic<bool> cancel_requested{false};
        bool cancel_sent = false;
        // budget bytes a finished job keeps until it is released: a render the
        // server created keeps its images and pixel state
        long long held = 0;
};

Server::Server(const int max_jobs, const long long memory_budget)
        : max_jobs_(max_jobs),
          budget_(memory_budget),
          start_(steady_seconds())
{
        if (max_jobs < 1)
        {
                throw std::runtime_error("server needs at least one job slot");
        }
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess)
        {
                cudaGetLastError();
                throw std::runtime_error("no CUDA device for the server");
        }
        if (memory_budget <= 0)
        {
                std::size_t free = 0;
                std::size_t total = 0;
                if (cudaMemGetInfo(&free, &total) != cudaSuccess)
                {
                        cudaGetLastError();
                        throw std::runtime_error("no CUDA device for the server");
                }
                budget_ = static_cast<long long>(free * 0.8);
        }
        initial_budget_ = budget_;
        {
                cudaEvent_t e = nullptr;
                cuda_check(cudaEventCreate(&e), "cudaEventCreate");
                reference_event_ = e;
                cuda_check(cudaEventRecord(e, nullptr), "cudaEventRecord");
        }
        {
                // registered after the CUDA runtime initialised above, so it
                // runs before the runtime's own exit handlers
                const std::lock_guard lock(g_live_mutex);
                if (!g_live)
                {
                        g_live = new std::set<Server*>;
                        std::atexit(stop_live_servers);
                }
                g_live->insert(this);
        }
        worker_ = std::thread(&Server::run, this);
}

void Server::shutdown()
{
        {
                const std::lock_guard lock(mutex_);
                stop_ = true;
        }
        changed_.notify_all();
        if (worker_.joinable() && worker_.get_id() != std::this_thread::get_id())
        {
                worker_.join();
        }
}

Server::~Server()
{
        shutdown();
        if (reference_event_)
        {
                cudaEventDestroy(static_cast<cudaEvent_t>(reference_event_));
        }
        const std::lock_guard lock(g_live_mutex);
        if (g_live)
        {
                g_live->erase(this);
        }
}

double Server::now() const
{
        return steady_seconds() - start_;
}

long long Server::submit(Painter* const painter, const int passes)
{
        if (!painter)
        {
                throw std::runtime_error("null painter");
        }
        if (passes < 1)
        {
                throw std::runtime_error("a job needs at least one pass");
        }
        auto job = std::make_shared<Job>();
        job->painter = painter;
        if (cudaGetDevice(&job->device) != cudaSuccess)
        {
                cudaGetLastError();
                throw std::runtime_error("no CUDA device for the job");
        }
        job->info.state = JobState::QUEUED;
        job->info.passes = passes;
        job->info.passes_done = 0;
        job->info.footprint = painter->device_bytes();
        job->info.submitted = now();
        job->info.started = -1;
        job->info.finished = -1;
        long long id = 0;
        {
                const std::lock_guard lock(mutex_);
                if (stop_)
                {
                        throw std::runtime_error("the server is stopping");
                }
                id = next_id_++;
                job->id = id;
                jobs_[id] = job;
                queue_.push_back(job);
        }
        changed_.notify_all();
        return id;
}

long long Server::submit_render(Scene* const scene, const int spp, const int max_depth, const std::uint32_t seed,
                               const int passes)
{
        if (!scene)
        {
                throw std::runtime_error("null scene");
        }
        if (passes < 1)
        {
                throw std::runtime_error("a job needs at least one pass");
        }
        auto job = std::make_shared<Job>();
        job->scene = scene;
        job->spp = spp;
        job->max_depth = max_depth;
        job->seed = seed;
        if (cudaGetDevice(&job->device) != cudaSuccess)
        {
                cudaGetLastError();
                throw std::runtime_error("no CUDA device for the job");
        }
        job->info.state = JobState::QUEUED;
        job->info.passes = passes;
        job->info.passes_done = 0;
        {
                const std::lock_guard lock(mutex_);
                job->chunk_budget = slot_chunk_budget();
        }
        job->info.footprint =
                scene->painter_bytes(spp, max_depth, Integrator::BPT, job->chunk_budget) + scene->device_bytes();
        job->info.submitted = now();
        job->info.started = -1;
        job->info.finished = -1;
        long long id = 0;
        {
                const std::lock_guard lock(mutex_);
                if (stop_)
                {
                        throw std::runtime_error("the server is stopping");
                }
                id = next_id_++;
                job->id = id;
                jobs_[id] = job;
                queue_.push_back(job);
        }
        changed_.notify_all();
        return id;
}

std::shared_ptr<Server::Job> Server::find_locked(const long long job) const
{
        const auto i = jobs_.find(job);
        if (i == jobs_.end())
        {
                throw std::runtime_error("unknown job " + std::to_string(job));
        }
        return i->second;
}

JobInfo Server::info(const long long job) const
{
        const std::lock_guard lock(mutex_);
        return find_locked(job)->info;
}

void Server::images(const long long job, float* const rgb, float* const rgba)
{
        std::shared_ptr<Job> j;
        {
                const std::lock_guard lock(mutex_);
                j = find_locked(job);
                if (j->info.state != JobState::DONE)
                {
                        throw std::runtime_error("job " + std::to_string(job) + " is not done");
                }
        }
        cudaSetDevice(j->device);
        j->painter->images(rgb, rgba);
}

Statistics Server::statistics(const long long job)
{
        std::shared_ptr<Job> j;
        {
                const std::lock_guard lock(mutex_);
                j = find_locked(job);
                if (j->info.state != JobState::DONE)
                {
                        throw std::runtime_error("job " + std::to_string(job) + " is not done");
                }
        }
        return j->painter->statistics();
}

void Server::release(const long long job)
{
        std::shared_ptr<Job> j;
        {
                const std::lock_guard lock(mutex_);
                j = find_locked(job);
                if (j->info.state != JobState::DONE && j->info.state != JobState::FAILED)
                {
                        throw std::runtime_error("job " + std::to_string(job) + " is not finished");
                }
                jobs_.erase(job);
                used_ -= j->held;
                j->held = 0;
        }
        if (j->owned)
        {
                cudaSetDevice(j->device);
                j->owned.reset();
        }
        changed_.notify_all();
}

JobInfo Server::wait(const long long job)
{
        std::unique_lock lock(mutex_);
        const std::shared_ptr<Job> j = find_locked(job);
        changed_.wait(lock,
                      [&]
                      {
                              return j->info.state == JobState::DONE || j->info.state == JobState::FAILED;
                      });
        return j->info;
}

// Admits queued jobs in arrival order while a slot and the memory budget
// allow; a job larger than the whole budget is admitted when nothing runs.
bool Server::admit_locked()
{
        bool any = false;
        if (hold_)
        {
                return false;
        }
        while (!queue_.empty() && static_cast<int>(running_.size()) < max_jobs_)
        {
                const std::shared_ptr<Job>& j = queue_.front();
                if (!running_.empty() && used_ + j->info.footprint > budget_)
                {
                        break;
                }
                used_ += j->info.footprint;
                j->info.state = JobState::RUNNING;
                j->info.started = now();
                running_.push_back(j);
                queue_.pop_front();
                any = true;
        }
        return any;
}

void Server::finish_locked(Job& job, const JobState state, const std::string& error)
{
        job.info.state = state;
        job.info.error = error;
        job.info.finished = now();
        cudaSetDevice(job.device);
        // a render the server created keeps its images until it is released:
        // its per-chunk path buffers go back now, the rest stays counted
        long long freed = job.info.footprint;
        if (job.owned)
        {
                try
                {
                        freed = std::min(job.info.footprint, job.owned->release_scratch());
                }
                catch (const std::exception&)
                {
                        cudaGetLastError();
                        freed = 0;
                }
        }
        job.held = job.info.footprint - freed;
        used_ -= freed;
        budget_ = initial_budget_; // memory freed: admit by the estimate again
        if (state == JobState::DONE && job.first && job.done)
        {
                const cudaEvent_t reference = static_cast<cudaEvent_t>(reference_event_);
                float a = 0;
                float b = 0;
                if (cudaEventElapsedTime(&a, reference, job.first) == cudaSuccess &&
                    cudaEventElapsedTime(&b, reference, job.done) == cudaSuccess)
                {
                        job.info.device_started = a * 1e-3;
                        job.info.device_finished = b * 1e-3;
                }
                else
                {
                        cudaGetLastError();
                }
        }
        for (cudaEvent_t* e : {&job.first, &job.done})
        {
                if (*e)
                {
                        cudaEventDestroy(*e);
                        *e = nullptr;
                }
        }
}

void Server::cancel(const long long job)
{
        {
                const std::lock_guard lock(mutex_);
                const std::shared_ptr<Job> j = find_locked(job);
                if (j->info.state == JobState::QUEUED)
                {
                        for (auto i = queue_.begin(); i != queue_.end(); ++i)
                        {
                                if (i->get() == j.get())
                                {
                                        queue_.erase(i);
                                        break;
                                }
                        }
                        // a queued job holds no device memory or budget
                        j->info.state = JobState::FAILED;
                        j->info.error = "cancelled";
                        j->info.finished = now();
                }
                else if (j->info.state == JobState::RUNNING)
                {
                        j->cancel_requested = true;
                }
        }
        changed_.notify_all();
}

void Server::fail_next_creations(const int count)
{
        const std::lock_guard lock(mutex_);
        fail_creations_ = count;
}

// The chunk buffers of a render the server creates: an equal share of the
// memory budget per slot, so that max_jobs renders fit at once, and at least
// 4 GiB.  Running jobs overlap one another's chunk tails, so smaller chunks
// cost less here than in a render alone.
long long Server::slot_chunk_budget() const
{
        if (chunk_budget_ > 0)
        {
                return chunk_budget_;
        }
        return std::max(4LL << 30, initial_budget_ / std::max(1, max_jobs_));
}

void Server::set_chunk_budget(const long long bytes)
{
        if (bytes < 0)
        {
                throw std::runtime_error("chunk budget " + std::to_string(bytes) + " is negative");
        }
        const std::lock_guard lock(mutex_);
        chunk_budget_ = bytes;
}

long long Server::chunk_budget() const
{
        const std::lock_guard lock(mutex_);
        return slot_chunk_budget();
}

void Server::hold_admission(const bool hold)
{
        {
                const std::lock_guard lock(mutex_);
                hold_ = hold;
        }
        changed_.notify_all();
}

// The worker keeps one pass of every running job in flight, on the job's own
// stream, and retires passes as their events complete.
void Server::run()
{
        while (true)
        {
                std::deque<std::shared_ptr<Job>> running;
                {
                        std::unique_lock lock(mutex_);
                        if (stop_ && running_.empty())
                        {
                                for (const std::shared_ptr<Job>& j : queue_)
                                {
                                        j->info.state = JobState::FAILED;
                                        j->info.error = "server stopped";
                                        j->info.finished = now();
                                }
                                queue_.clear();
                                changed_.notify_all();
                                return;
                        }
                        if (!stop_)
                        {
                                admit_locked();
                        }
                        if (running_.empty())
                        {
                                changed_.wait_for(lock, std::chrono::milliseconds(5));
                                continue;
                        }
                        running = running_;
                }

                bool progressed = false;
                // renders whose creation ran out of device memory go back to the
                // head of the queue in their admission (= arrival) order
                std::size_t returned = 0;
                for (const std::shared_ptr<Job>& j : running)
                {
                        std::string error;
                        bool finished = false;
                        try
                        {
                                cudaSetDevice(j->device);
                                if (!j->painter && j->cancel_requested)
                                {
                                        throw std::runtime_error("cancelled");
                                }
                                if (!j->painter)
                                {
                                        // a render created at admission
                                        try
                                        {
                                                bool fail = false;
                                                {
                                                        const std::lock_guard lock(mutex_);
                                                        if (fail_creations_ > 0)
                                                        {
                                                                --fail_creations_;
                                                                fail = true;
                                                        }
                                                }
                                                if (fail)
                                                {
                                                        throw CudaError("cudaMalloc (a failure the test asked for)",
                                                                        cudaErrorMemoryAllocation);
                                                }
                                                j->owned = j->scene->create_painter(j->spp, j->max_depth, j->seed,
                                                                                    Integrator::BPT, 0, -1, false,
                                                                                    j->chunk_budget);
                                        }
                                        catch (const CudaError& e)
                                        {
                                                if (e.code() != cudaErrorMemoryAllocation)
                                                {
                                                        throw;
                                                }
                                                cudaGetLastError();
                                                // the estimate let in more than the device holds: back to
                                                // the head of the queue, and admit no more than what runs
                                                // now until a job ends
                                                const std::lock_guard lock(mutex_);
                                                if (running_.size() <= 1)
                                                {
                                                        throw;
                                                }
                                                for (auto i = running_.begin(); i != running_.end(); ++i)
                                                {
                                                        if (i->get() == j.get())
                                                        {
                                                                running_.erase(i);
                                                                break;
                                                        }
                                                }
                                                used_ -= j->info.footprint;
                                                j->info.state = JobState::QUEUED;
                                                j->info.started = -1;
                                                queue_.insert(queue_.begin() + static_cast<std::ptrdiff_t>(returned), j);
                                                ++returned;
                                                budget_ = used_;
                                                continue;
                                        }
                                        j->painter = j->owned.get();
                                }
                                if (j->cancel_requested)
                                {
                                        if (j->pass_in_flight)
                                        {
                                                if (!j->cancel_sent)
                                                {
                                                        j->painter->cancel();
                                                        j->cancel_sent = true;
                                                }
                                                const cudaError_t e = cudaEventQuery(j->done);
                                                if (e == cudaErrorNotReady)
                                                {
                                                        continue;
                                                }
                                                j->pass_in_flight = false;
                                        }
                                        throw std::runtime_error("cancelled");
                                }
                                if (j->pass_in_flight)
                                {
                                        const cudaError_t e = cudaEventQuery(j->done);
                                        if (e == cudaErrorNotReady)
                                        {
                                                continue;
                                        }
                                        if (e != cudaSuccess)
                                        {
                                                throw CudaError("pass failed", e);
                                        }
                                        j->pass_in_flight = false;
                                        progressed = true;
                                        {
                                                const std::lock_guard lock(mutex_);
                                                ++j->info.passes_done;
                                        }
                                        if (j->info.passes_done == j->info.passes)
                                        {
                                                j->painter->wait(); // statistics of the last pass
                                                finished = true;
                                        }
                                }
                                if (!finished && !j->pass_in_flight)
                                {
                                        if (!j->done)
                                        {
                                                cuda_check(cudaEventCreate(&j->done), "cudaEventCreate");
                                        }
                                        if (!j->first)
                                        {
                                                cuda_check(cudaEventCreate(&j->first), "cudaEventCreate");
                                                cuda_check(cudaEventRecord(j->first,
                                                                           static_cast<cudaStream_t>(j->painter->stream())),
                                                           "cudaEventRecord");
                                        }
                                        j->painter->enqueue_passes(1);
                                        cuda_check(cudaEventRecord(j->done, static_cast<cudaStream_t>(j->painter->stream())),
                                                   "cudaEventRecord");
                                        j->pass_in_flight = true;
                                        progressed = true;
                                }
                        }
                        catch (const std::exception& e)
                        {
                                error = e.what();
                                cudaGetLastError();
                        }
                        if (finished || !error.empty())
                        {
                                const std::lock_guard lock(mutex_);
                                finish_locked(*j, error.empty() ? JobState::DONE : JobState::FAILED, error);
                                for (auto i = running_.begin(); i != running_.end(); ++i)
                                {
                                        if (i->get() == j.get())
                                        {
                                                running_.erase(i);
                                                break;
                                        }
                                }
                                admit_locked();
                                changed_.notify_all();
                        }
                }
                if (!progressed)
                {
                        std::this_thread::sleep_for(std::chrono::microseconds(50));
                }
        }
}
} // namespace nbpt
