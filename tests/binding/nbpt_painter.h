// The reference-side binding of nbpt: a painter::Painter that renders
// through the C ABI (include/nbpt.h) instead of the CPU painter, as a
// maintainer would add it to src/painter/ and choose it in create_painter
// (src/painter/painter.cpp:136-157) when a GPU is present.  Compiled against
// the reference's own headers by oracle/Makefile and run by
// tests/test_binding.py.
//
// The library runs the passes on its own worker thread and hands each pass's
// images to a callback, as the reference's painter thread calls its
// Notifier (src/painter/painter.cpp:77-134, painter.h:36-118), so the binding
// only copies the images into the notifier's Images under ImagesWriting, in
// the layout Pixels::images writes (src/painter/pixels/pixels.cpp:123-166).
#pragma once

#include "../../include/nbpt.h"

#include <src/com/error.h>
#include <src/painter/painter.h>

#include <array>
#include <cstddef>
#include <cstring>
#include <optional>
#include <string>

namespace ns::painter
{
template <std::size_t N>
class NbptPainter final : public Painter
{
        static constexpr std::size_t RGB_PIXEL_SIZE = 3 * sizeof(float);
        static constexpr std::size_t RGBA_PIXEL_SIZE = 4 * sizeof(float);

        Notifier<N - 1>* notifier_;
        std::array<int, N - 1> screen_size_;
        nbpt_painter* painter_ = nullptr;

        // the library's worker thread, after every pass; `pass` counts from
        // 1, as the reference's Statistics::pass_number does
        static void on_pass(void* user, long long pass, const float* rgb, const float* rgba, long long pixels)
        {
                auto* const self = static_cast<NbptPainter*>(user);
                {
                        const ImagesWriting lock(self->notifier_->images(pass));
                        image::Image<N - 1>& with_background = lock.image_with_background();
                        with_background.color_format = image::ColorFormat::R32G32B32;
                        with_background.size = self->screen_size_;
                        with_background.pixels.resize(RGB_PIXEL_SIZE * pixels);
                        std::memcpy(with_background.pixels.data(), rgb, RGB_PIXEL_SIZE * pixels);
                        image::Image<N - 1>& without_background = lock.image_without_background();
                        without_background.color_format = image::ColorFormat::R32G32B32A32_PREMULTIPLIED;
                        without_background.size = self->screen_size_;
                        without_background.pixels.resize(RGBA_PIXEL_SIZE * pixels);
                        std::memcpy(without_background.pixels.data(), rgba, RGBA_PIXEL_SIZE * pixels);
                }
                self->notifier_->pass_done(pass);
        }

        // errors during painting go to the notifier and end the painting
        // (src/painter/painting/painting.cpp:121-164)
        static void on_error(void* user, const char* message)
        {
                static_cast<NbptPainter*>(user)->notifier_->error_message(std::string("Painter error:\n") + message);
        }

public:
        // max_depth is the reference's MAX_DEPTH (src/painter/integrators/bpt/bpt.cpp:58)
        NbptPainter(const Integrator integrator,
                    Notifier<N - 1>* const notifier,
                    nbpt_scene* const scene,
                    const std::array<int, N - 1>& screen_size,
                    const int samples_per_pixel,
                    const std::optional<int> max_pass_count,
                    const int max_depth = 5,
                    const unsigned seed = 1)
                : notifier_(notifier),
                  screen_size_(screen_size)
        {
                // invalid arguments throw synchronously (src/painter/painter.cpp:41-73)
                if (!notifier)
                {
                        error("Painter notifier is null");
                }
                if (max_pass_count && *max_pass_count < 1)
                {
                        error("Painter maximum pass count (" + std::to_string(*max_pass_count) +
                              ") must be greater than 0");
                }
                painter_ = nbpt_painter_create_integrator(
                        scene, integrator == Integrator::PT ? NBPT_INTEGRATOR_PT : NBPT_INTEGRATOR_BPT,
                        samples_per_pixel, max_depth, seed);
                if (!painter_)
                {
                        error(nbpt_last_error());
                }
                if (nbpt_painter_start(painter_, max_pass_count.value_or(0), on_pass, on_error, this) < 0)
                {
                        const std::string message = nbpt_last_error();
                        nbpt_painter_destroy(painter_);
                        error(message);
                }
        }

        NbptPainter(const NbptPainter&) = delete;
        NbptPainter& operator=(const NbptPainter&) = delete;

        // as the reference's destructor: stop (the pass in flight takes no
        // more paths) and join (src/painter/painter.cpp:129-134)
        ~NbptPainter() override
        {
                nbpt_painter_cancel(painter_);
                nbpt_painter_join(painter_);
                nbpt_painter_destroy(painter_);
        }

        void wait() noexcept override
        {
                nbpt_painter_join(painter_);
        }

        // answers after wait(): while the worker runs the painter's other calls fail
        [[nodiscard]] Statistics statistics() const override
        {
                nbpt_statistics s{};
                Statistics r;
                r.pass_number = 0;
                r.pass_progress = 0;
                r.pixel_count = 0;
                r.ray_count = 0;
                r.sample_count = 0;
                r.previous_pass_duration = 0;
                if (nbpt_painter_statistics(painter_, &s) == NBPT_OK)
                {
                        r.pass_number = s.pass_number;
                        r.pixel_count = s.pixel_count;
                        r.ray_count = s.ray_count;
                        r.sample_count = s.sample_count;
                        r.previous_pass_duration = s.previous_pass_duration;
                }
                return r;
        }
};
}
