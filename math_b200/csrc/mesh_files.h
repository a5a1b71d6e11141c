// n-dimensional mesh files: OBJ (v, vn, f, usemtl, mtllib with Kd) and STL
// (ASCII and binary), read as the reference's loaders read them
// (src/model/mesh/file/load_obj.cpp, obj/*.cpp, load_stl.cpp, mesh_facet.h).
#pragma once

#include <array>
#include <string>
#include <vector>

namespace nbpt::host
{
struct MeshFile final
{
        int n = 0;
        std::vector<float> vertices;         // [V][n]
        std::vector<float> normals;          // [M][n], unit or zero
        std::vector<int> facet_vertices;     // [F][n]
        std::vector<int> facet_normals;      // [F][n], -1 where the facet has none
        std::vector<unsigned char> has_normal; // [F]
        std::vector<int> facet_material;     // [F], -1: the object's own colour
        std::vector<std::array<float, 3>> material_colors; // Kd of each used material
};

// The file's dimension from its name: .obj / .stl are 3-space, .objN / .stlN
// N-space (src/model/mesh/file/file_type.cpp); 0 when neither.
int mesh_file_dimension(const std::string& path);

// Reads an OBJ or STL file of dimension n (3, 4 or 5); throws with the
// reference's messages on malformed input.
MeshFile load_mesh_file(const std::string& path, int n);
} // namespace nbpt::host
