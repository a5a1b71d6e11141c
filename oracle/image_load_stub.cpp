// Build-side stub: the reference reads OBJ material texture images through
// Qt (src/image/file_load.cpp), which this image lacks.  The oracle's mesh
// files carry no textures; a file that names one fails here.
#include <src/image/file_load.h>

#include <filesystem>
#include <stdexcept>

namespace ns::image
{
template <typename Path>
Image<2> load_rgba(const Path&)
{
        throw std::runtime_error("Texture images are not supported");
}

template Image<2> load_rgba(const std::filesystem::path&);
} // namespace ns::image
