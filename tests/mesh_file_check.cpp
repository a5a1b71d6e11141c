// Reads an n-dimensional OBJ or STL file with the library's loader
// (math_b200/csrc/mesh_files.cpp) and writes what it read to a binary file
// for tests/test_mesh_files.py: the vertex, normal and facet counts (three
// int64), then the vertices [V][n] and normals [M][n] as float32, the
// facets' vertex and normal indices [F][n] as int32, has_normal [F] as
// uint8 and the facets' materials [F] as int32.
//
//   mesh_file_check <file> <n> <output>

#include "mesh_files.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <vector>

namespace
{
template <typename T>
void put(std::FILE* const out, const std::vector<T>& v)
{
        if (!v.empty())
        {
                std::fwrite(v.data(), sizeof(T), v.size(), out);
        }
}
} // namespace

int main(const int argc, char** const argv)
{
        if (argc != 4)
        {
                std::fprintf(stderr, "usage: mesh_file_check <file> <n> <output>\n");
                return 2;
        }
        try
        {
                const int n = std::atoi(argv[2]);
                const nbpt::host::MeshFile m = nbpt::host::load_mesh_file(argv[1], n);
                std::FILE* const out = std::fopen(argv[3], "wb");
                if (out == nullptr)
                {
                        std::fprintf(stderr, "cannot write %s\n", argv[3]);
                        return 1;
                }
                const std::int64_t counts[3] = {static_cast<std::int64_t>(m.vertices.size() / n),
                                                static_cast<std::int64_t>(m.normals.size() / n),
                                                static_cast<std::int64_t>(m.has_normal.size())};
                std::fwrite(counts, sizeof(counts[0]), 3, out);
                put(out, m.vertices);
                put(out, m.normals);
                put(out, m.facet_vertices);
                put(out, m.facet_normals);
                put(out, m.has_normal);
                put(out, m.facet_material);
                std::fclose(out);
        }
        catch (const std::exception& e)
        {
                std::fprintf(stderr, "%s\n", e.what());
                return 1;
        }
        return 0;
}
