// Scene and painter instantiations for 5-space.
#include "painter_impl.cuh"

namespace nbpt
{
std::unique_ptr<Scene> make_scene_5(const bool double_precision, const bool spectrum)
{
        return make_scene_n<5>(double_precision, spectrum);
}
} // namespace nbpt
