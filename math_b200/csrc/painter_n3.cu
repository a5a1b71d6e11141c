// Scene and painter instantiations for 3-space.
#include "painter_impl.cuh"

namespace nbpt
{
std::unique_ptr<Scene> make_scene_3(const bool double_precision, const bool spectrum)
{
        return make_scene_n<3>(double_precision, spectrum);
}
} // namespace nbpt
