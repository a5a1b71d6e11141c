// Drives the reference-side binding (nbpt_painter.h) with a test Notifier
// that records every call, on a 3-space box built through the C ABI, and
// checks that: passes are numbered 1, 2, 3 with images before each
// pass_done; the notifier's images equal a C-ABI painter's with the same
// seed and passes; invalid arguments throw synchronously; an unbounded
// painter destroyed mid-render stops; errors reach error_message.  Prints
// "binding ok" and exits 0, or prints the failure and exits 1.
#include "nbpt_painter.h"

#include <src/painter/painter.h>

#include <array>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace
{
using ns::painter::Images;
using ns::painter::ImagesReading;

class RecordingNotifier final : public ns::painter::Notifier<2>
{
        Images<2> images_;

public:
        std::mutex mutex;
        std::vector<long long> images_calls;
        std::vector<long long> pass_done_calls;
        std::vector<std::string> errors;

        void thread_busy(unsigned, const std::array<int, 2>&) override
        {
        }
        void thread_free(unsigned) override
        {
        }
        void pixel_set(const std::array<int, 2>&, const ns::numerical::Vector<3, float>&) override
        {
        }
        Images<2>* images(const long long pass) override
        {
                const std::lock_guard lock(mutex);
                images_calls.push_back(pass);
                return &images_;
        }
        void pass_done(const long long pass) override
        {
                const std::lock_guard lock(mutex);
                pass_done_calls.push_back(pass);
        }
        void error_message(const std::string& msg) override
        {
                const std::lock_guard lock(mutex);
                errors.push_back(msg);
        }

        std::vector<float> rgb() const
        {
                const ImagesReading<2> lock(&images_);
                const auto& image = lock.image_with_background();
                std::vector<float> out(image.pixels.size() / sizeof(float));
                std::memcpy(out.data(), image.pixels.data(), image.pixels.size());
                return out;
        }
};

void check(const bool ok, const std::string& what)
{
        if (!ok)
        {
                throw std::runtime_error(what);
        }
}

// the C ABI's status: negative on failure (the add_* calls return an index)
void ok(const int status)
{
        check(status >= 0, std::string("C ABI call failed: ") + nbpt_last_error());
}

constexpr std::array<int, 2> SCREEN{24, 20};

// a box of five 2x2 walls open towards the camera, a ceiling light and a
// rotated solid parallelotope, finalized in double precision
nbpt_scene* make_scene()
{
        nbpt_scene* s = nbpt_scene_create(3, NBPT_DOUBLE, NBPT_RGB);
        check(s != nullptr, nbpt_last_error());
        const float grey[3] = {0.7f, 0.7f, 0.7f};
        const float red[3] = {0.7f, 0.1f, 0.1f};
        struct Wall
        {
                double org[3];
                double v[6];
                const float* color;
        };
        const Wall walls[] = {
                {{-1, -1, -1}, {0, 2, 0, 0, 0, 2}, red},   // x = -1
                {{1, -1, -1}, {0, 0, 2, 0, 2, 0}, grey},   // x = +1
                {{-1, -1, -1}, {0, 0, 2, 2, 0, 0}, grey},  // y = -1
                {{-1, 1, -1}, {2, 0, 0, 0, 0, 2}, grey},   // y = +1
                {{-1, -1, 1}, {2, 0, 0, 0, 2, 0}, grey},   // z = +1
        };
        for (const Wall& w : walls)
        {
                ok(nbpt_scene_add_hyperplane_parallelotope(s, 0, 1, w.color, 1, w.org, w.v));
        }
        const double light_org[3] = {-0.25, 0.99, -0.25};
        const double light_v[6] = {0.5, 0, 0, 0, 0, 0.5};
        const float white[3] = {1, 1, 1};
        ok(nbpt_scene_add_hyperplane_parallelotope(s, 0, 1, white, 1, light_org, light_v));
        const double down[3] = {0, -1, 0};
        const float radiance[3] = {10, 10, 10};
        ok(nbpt_scene_add_parallelotope_light(s, 5, down, radiance));
        const double box_org[3] = {-0.3, -1, 0};
        const double box_v[9] = {0.4, 0, 0.2, 0, 0.6, 0, -0.2, 0, 0.4};
        const float gold[3] = {0.8f, 0.6f, 0.3f};
        ok(nbpt_scene_add_parallelotope(s, 1, 0.3, gold, 1, box_org, box_v));
        const double org[3] = {0, 0, -3};
        const double dir[3] = {0, 0, 1};
        const double axes[6] = {1, 0, 0, 0, 1, 0};
        ok(nbpt_scene_set_perspective_projector(s, org, dir, axes, 60, SCREEN.data()));
        const float black[3] = {0, 0, 0};
        ok(nbpt_scene_set_background(s, black));
        ok(nbpt_scene_finalize(s));
        return s;
}

void run()
{
        nbpt_scene* const scene = make_scene();
        const long long pixels = nbpt_scene_pixel_count(scene);
        constexpr int SPP = 16;
        constexpr int PASSES = 3;

        // the images of three passes through the binding
        RecordingNotifier notifier;
        {
                ns::painter::NbptPainter<3> painter(
                        ns::painter::Integrator::BPT, &notifier, scene, SCREEN, SPP, PASSES, 5, 7);
                painter.wait();
                const ns::painter::Statistics st = painter.statistics();
                check(st.pass_number == PASSES, "statistics: pass number");
                check(st.pixel_count == pixels, "statistics: pixel count");
                check(st.sample_count == pixels * SPP, "statistics: sample count");
        }
        check(notifier.pass_done_calls == std::vector<long long>{1, 2, 3}, "pass_done must be called for passes 1, 2, 3");
        check(notifier.images_calls == std::vector<long long>{1, 2, 3}, "images must be asked for passes 1, 2, 3");
        check(notifier.errors.empty(), "no error expected");

        // the same render through the C ABI directly
        nbpt_painter* direct = nbpt_painter_create(scene, SPP, 5, 7);
        check(direct != nullptr, nbpt_last_error());
        ok(nbpt_painter_enqueue(direct, PASSES));
        ok(nbpt_painter_wait(direct));
        std::vector<float> rgb(pixels * 3);
        ok(nbpt_painter_images(direct, rgb.data(), nullptr));
        nbpt_painter_destroy(direct);
        check(notifier.rgb() == rgb, "the notifier's image differs from the C ABI painter's");

        // invalid arguments throw synchronously, as create_painter does
        bool thrown = false;
        try
        {
                RecordingNotifier n;
                ns::painter::NbptPainter<3> bad(ns::painter::Integrator::BPT, &n, scene, SCREEN, 0, 1);
        }
        catch (const std::exception&)
        {
                thrown = true;
        }
        check(thrown, "samples per pixel 0 must throw");
        thrown = false;
        try
        {
                RecordingNotifier n;
                ns::painter::NbptPainter<3> bad(ns::painter::Integrator::BPT, &n, scene, SCREEN, SPP, 0);
        }
        catch (const std::exception&)
        {
                thrown = true;
        }
        check(thrown, "maximum pass count 0 must throw");

        // an unbounded painter (no maximum pass count) ends when destroyed
        {
                RecordingNotifier n;
                {
                        ns::painter::NbptPainter<3> endless(
                                ns::painter::Integrator::PT, &n, scene, SCREEN, SPP, std::nullopt);
                        while (true)
                        {
                                {
                                        const std::lock_guard lock(n.mutex);
                                        if (n.pass_done_calls.size() >= 2)
                                        {
                                                break;
                                        }
                                }
                                std::this_thread::yield();
                        }
                }
                check(n.pass_done_calls.size() >= 2, "the endless painter must have run passes");
                for (std::size_t i = 0; i < n.pass_done_calls.size(); ++i)
                {
                        check(n.pass_done_calls[i] == static_cast<long long>(i) + 1, "passes numbered from 1");
                }
        }
        nbpt_scene_destroy(scene);
}
} // namespace

int main()
{
        try
        {
                run();
        }
        catch (const std::exception& e)
        {
                std::printf("binding check failed: %s\n", e.what());
                return 1;
        }
        std::printf("binding ok\n");
        return 0;
}
