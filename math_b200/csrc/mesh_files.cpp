#include "mesh_files.h"

#include <algorithm>
#include <array>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <thread>
#include <vector>

namespace nbpt::host
{
namespace
{
[[noreturn]] void fail(const std::string& message)
{
        throw std::runtime_error(message);
}

std::vector<char> read_bytes(const std::filesystem::path& path)
{
        std::ifstream f(path, std::ios::binary);
        if (!f)
        {
                fail("Failed to open file " + path.generic_string());
        }
        f.seekg(0, std::ios::end);
        const std::streamoff size = f.tellg();
        f.seekg(0, std::ios::beg);
        std::vector<char> data(static_cast<std::size_t>(size));
        if (size > 0 && !f.read(data.data(), size))
        {
                fail("Failed to read file " + path.generic_string());
        }
        return data;
}

// src/com/string/ascii.h
bool is_space(const char c)
{
        return c == ' ' || (c <= '\x0d' && c >= '\x09');
}

bool is_print(const char c)
{
        return c >= '\x20' && c <= '\x7e';
}

// What strtof reads (leading white space, an optional sign, decimal,
// hexadecimal, infinity or NaN forms), with the reference's checks
// (src/com/read.h): a number must be read, and it must be finite.  Decimal
// numbers go through std::from_chars, which rounds as strtof does.
bool read_float(const char*& s, float& out)
{
        const char* p = s;
        while (*p && is_space(*p))
        {
                ++p;
        }
        const char* q = (*p == '+' && p[1] != '+' && p[1] != '-') ? p + 1 : p;
        // the characters a number can be made of; the text ends with a zero
        const char* line_end = q;
        while (std::isalnum(static_cast<unsigned char>(*line_end)) || *line_end == '.' || *line_end == '+' ||
               *line_end == '-' || *line_end == '(' || *line_end == ')' || *line_end == '_')
        {
                ++line_end;
        }
        float v = 0;
        const auto [ptr, ec] = std::from_chars(q, line_end, v);
        const bool hex = ptr < line_end && (*ptr == 'x' || *ptr == 'X');
        const char* end = ptr;
        if (hex || ec == std::errc::result_out_of_range || (ec != std::errc{} && ptr != q))
        {
                char* e = nullptr;
                v = std::strtof(s, &e);
                end = e;
        }
        else if (ec != std::errc{})
        {
                end = s;
        }
        if (end <= s)
        {
                return false;
        }
        if (!std::isfinite(v))
        {
                fail("Error reading float");
        }
        out = v;
        s = end;
        return true;
}

void read_floats(const char*& s, float* out, const int count)
{
        for (int i = 0; i < count; ++i)
        {
                if (!read_float(s, out[i]))
                {
                        fail("Error reading vector data");
                }
        }
}

// ---------------------------------------------------------------------------
// text lines (src/model/mesh/file/lines.cpp, obj/data_read.cpp)

struct Lines final
{
        std::vector<char> data;
        std::vector<std::size_t> begin;

        explicit Lines(std::vector<char>&& text)
                : data(std::move(text))
        {
                if (data.empty())
                {
                        return;
                }
                if (data.back() != '\n')
                {
                        data.push_back('\n');
                }
                std::size_t start = 0;
                for (std::size_t i = 0; i < data.size(); ++i)
                {
                        if (data[i] == '\0')
                        {
                                fail("Text data contains null character");
                        }
                        if (data[i] == '\n')
                        {
                                data[i] = '\0';
                                begin.push_back(start);
                                start = i + 1;
                        }
                }
        }

        std::size_t size() const
        {
                return begin.size();
        }

        // the line without its terminator
        std::string_view line(const std::size_t i) const
        {
                const char* const b = data.data() + begin[i];
                return {b, std::strlen(b)};
        }
};

// keyword and the rest of the line up to a comment
struct Split final
{
        std::string_view first;
        const char* rest_b;
        const char* rest_e;
};

Split split(const std::string_view line)
{
        const char* p = line.data();
        const char* const last = line.data() + line.size();
        while (p < last && is_space(*p))
        {
                ++p;
        }
        if (p == last || *p == '#')
        {
                return {{p, 0}, p, p};
        }
        const char* q = p + 1;
        while (q < last && !is_space(*q) && *q != '#')
        {
                ++q;
        }
        if (q == last || *q == '#')
        {
                return {{p, static_cast<std::size_t>(q - p)}, q, q};
        }
        const char* e = q;
        while (e < last && *e != '#')
        {
                ++e;
        }
        return {{p, static_cast<std::size_t>(q - p)}, q, e};
}

std::string_view read_name(const char* const what, const char* b, const char* const e)
{
        while (b < e && is_space(*b))
        {
                ++b;
        }
        if (b == e)
        {
                fail(std::string("Error read ") + what + " name");
        }
        const char* n = b;
        while (n < e && !is_space(*n))
        {
                ++n;
        }
        const char* r = n;
        while (r < e && is_space(*r))
        {
                ++r;
        }
        if (r != e)
        {
                fail(std::string("Error read ") + what + " name");
        }
        return {b, static_cast<std::size_t>(n - b)};
}

// ---------------------------------------------------------------------------
// OBJ (src/model/mesh/file/load_obj.cpp, obj/line.cpp, obj/facet.h,
// obj/line_process.h, obj/load_lib.cpp)

struct Corner final
{
        int vertex;
        int texcoord;
        int normal;
};

// "v", "v/t", "v/t/n", "v//n", "v/t/", "v//": the texture and normal
// indices are 0 when absent
const char* read_corner(const char* p, const char* const last, Corner& c)
{
        {
                int v = 0;
                const auto [ptr, ec] = std::from_chars(p, last, v);
                if (ec != std::errc{})
                {
                        if (ptr == p)
                        {
                                fail("Error read facet vertex first number");
                        }
                        fail("Error reading integral");
                }
                if (v == 0)
                {
                        fail("Zero facet index");
                }
                c.vertex = v;
                p = ptr;
        }
        int* const optional[2] = {&c.texcoord, &c.normal};
        for (int* const out : optional)
        {
                *out = 0;
                if (p == last || is_space(*p))
                {
                        continue;
                }
                if (*p != '/')
                {
                        fail(std::string("Error read facet number, expected '/', found '") + *p + "'");
                }
                ++p;
                if (p == last || is_space(*p))
                {
                        continue;
                }
                int v = 0;
                const auto [ptr, ec] = std::from_chars(p, last, v);
                if (ec != std::errc{})
                {
                        if (ptr == p)
                        {
                                continue; // no number: p stays on the next '/'
                        }
                        fail("Error reading integral");
                }
                if (v == 0)
                {
                        fail("Zero facet index");
                }
                *out = v;
                p = ptr;
        }
        return p;
}

// absolute index from 1-based (positive) or relative (negative) indices
int absolute_index(const int index, const int size)
{
        return index > 0 ? index - 1 : (index < 0 ? size + index : -1);
}

void read_color(const char* s, std::array<float, 3>& rgb)
{
        read_floats(s, rgb.data(), 3);
        for (const float x : rgb)
        {
                if (!(x >= 0 && x <= 1))
                {
                        fail("RGB components are not in the range [0, 1]");
                }
        }
}

enum class LineKind : unsigned char
{
        NONE,
        V,
        VT,
        VN,
        F,
        USEMTL,
        MTLLIB
};

// The lines of one part of an OBJ file, parsed: what does not depend on the
// lines before (numbers, normalised normals, facet corners) is read here, in
// parallel with the other parts.
struct ObjPart final
{
        std::vector<LineKind> kind;
        std::vector<float> values;               // v and vn payloads, n each
        std::vector<unsigned char> corner_count; // per f line
        std::vector<Corner> corners;
        std::size_t error_line = static_cast<std::size_t>(-1);
        std::string error;
};

void parse_obj_lines(const Lines& lines, const std::size_t begin, const std::size_t end, const int n,
                     const int max_corners, ObjPart& part)
{
        std::vector<Corner> corners(max_corners);
        std::vector<float> v(n);
        for (std::size_t i = begin; i < end; ++i)
        {
                const Split s = split(lines.line(i));
                try
                {
                        if (s.first == "v")
                        {
                                const char* p = s.rest_b;
                                read_floats(p, v.data(), n);
                                part.values.insert(part.values.end(), v.begin(), v.end());
                                part.kind.push_back(LineKind::V);
                        }
                        else if (s.first == "vt")
                        {
                                const char* p = s.rest_b;
                                read_floats(p, v.data(), n - 1);
                                float w = 0;
                                if (read_float(p, w) && !(w == 0))
                                {
                                        fail(std::to_string(n) + "-dimensional textures are not supported");
                                }
                                part.kind.push_back(LineKind::VT);
                        }
                        else if (s.first == "vn")
                        {
                                const char* p = s.rest_b;
                                read_floats(p, v.data(), n);
                                float sq = v[0] * v[0];
                                for (int k = 1; k < n; ++k)
                                {
                                        sq += v[k] * v[k];
                                }
                                const float norm = std::sqrt(sq);
                                bool finite = true;
                                for (float& x : v)
                                {
                                        x /= norm;
                                        finite = finite && std::isfinite(x);
                                }
                                if (!finite)
                                {
                                        std::fill(v.begin(), v.end(), 0.0f);
                                }
                                part.values.insert(part.values.end(), v.begin(), v.end());
                                part.kind.push_back(LineKind::VN);
                        }
                        else if (s.first == "f")
                        {
                                int count = 0;
                                const char* p = s.rest_b;
                                while (true)
                                {
                                        while (p < s.rest_e && is_space(*p))
                                        {
                                                ++p;
                                        }
                                        if (p == s.rest_e)
                                        {
                                                break;
                                        }
                                        if (count >= max_corners)
                                        {
                                                fail("Found too many facet vertices " + std::to_string(count + 1) +
                                                     " (max supported = " + std::to_string(max_corners) + ")");
                                        }
                                        p = read_corner(p, s.rest_e, corners[count]);
                                        ++count;
                                }
                                if (count < n)
                                {
                                        fail("Error facet vertex count " + std::to_string(count) + " (min = " +
                                             std::to_string(n) + ")");
                                }
                                int with_t = 0;
                                int with_n = 0;
                                for (int k = 0; k < count; ++k)
                                {
                                        with_t += corners[k].texcoord != 0 ? 1 : 0;
                                        with_n += corners[k].normal != 0 ? 1 : 0;
                                }
                                if (!(with_t == 0 || with_t == count))
                                {
                                        fail("Inconsistent facet texture indices");
                                }
                                if (!(with_n == 0 || with_n == count))
                                {
                                        fail("Inconsistent facet normal indices");
                                }
                                part.corner_count.push_back(static_cast<unsigned char>(count));
                                part.corners.insert(part.corners.end(), corners.begin(), corners.begin() + count);
                                part.kind.push_back(LineKind::F);
                        }
                        else if (s.first == "usemtl")
                        {
                                read_name("material", s.rest_b, s.rest_e);
                                part.kind.push_back(LineKind::USEMTL);
                        }
                        else if (s.first == "mtllib")
                        {
                                part.kind.push_back(LineKind::MTLLIB);
                        }
                        else
                        {
                                part.kind.push_back(LineKind::NONE);
                        }
                }
                catch (const std::exception& e)
                {
                        part.error_line = i;
                        part.error = "Line " + std::to_string(i) + ": " + std::string(s.first) + " " +
                                     std::string(s.rest_b, s.rest_e) + "\n" + e.what();
                        return;
                }
        }
}

void read_obj(const std::filesystem::path& path, const int n, MeshFile& m)
{
        const int max_corners = (n == 3 ? 5 : 1) + n - 1;
        std::vector<int> texcoord_index; // per facet corner, -1 without
        int texcoord_count = 0;
        int normal_count = 0;
        int material = -1;
        std::map<std::string, int, std::less<>> material_index; // materials still to find in the libraries
        std::vector<std::string> material_names;
        std::vector<std::filesystem::path> libraries;
        std::set<std::filesystem::path> unique_libraries;

        const Lines lines(read_bytes(path));

        // parse the lines in parts on the host threads, then apply them in order
        const std::size_t line_count = lines.size();
        const unsigned threads = static_cast<unsigned>(std::max<std::size_t>(
                1, std::min<std::size_t>(std::max(1u, std::thread::hardware_concurrency()), line_count / 4096)));
        std::vector<ObjPart> parts(threads);
        {
                std::vector<std::thread> pool;
                const std::size_t step = (line_count + threads - 1) / threads;
                for (unsigned t = 1; t < threads; ++t)
                {
                        pool.emplace_back(
                                [&, t]
                                {
                                        parse_obj_lines(lines, std::min(line_count, t * step),
                                                        std::min(line_count, (t + 1) * step), n, max_corners, parts[t]);
                                });
                }
                parse_obj_lines(lines, 0, std::min(line_count, step), n, max_corners, parts[0]);
                for (std::thread& th : pool)
                {
                        th.join();
                }
        }

        std::size_t i = 0;
        for (const ObjPart& part : parts)
        {
                std::size_t value = 0;
                std::size_t facet_line = 0;
                std::size_t corner = 0;
                for (const LineKind kind : part.kind)
                {
                        const std::size_t line = i++;
                        switch (kind)
                        {
                        case LineKind::NONE:
                                break;
                        case LineKind::V:
                                m.vertices.insert(m.vertices.end(), part.values.begin() + value,
                                                  part.values.begin() + value + n);
                                value += n;
                                break;
                        case LineKind::VT:
                                ++texcoord_count;
                                break;
                        case LineKind::VN:
                                m.normals.insert(m.normals.end(), part.values.begin() + value,
                                                 part.values.begin() + value + n);
                                value += n;
                                ++normal_count;
                                break;
                        case LineKind::F:
                        {
                                const int count = part.corner_count[facet_line++];
                                const Corner* const c0 = &part.corners[corner];
                                corner += count;
                                const int vertex_count = static_cast<int>(m.vertices.size() / n);
                                const bool normals = c0[0].normal != 0;
                                // a fan around the first corner
                                for (int f = 0; f + n - 1 < count; ++f)
                                {
                                        for (int k = 0; k < n; ++k)
                                        {
                                                const Corner& c = c0[k == 0 ? 0 : f + k];
                                                const int v = c.vertex > 0 ? c.vertex - 1 : vertex_count + c.vertex;
                                                m.facet_vertices.push_back(v);
                                                m.facet_normals.push_back(absolute_index(c.normal, normal_count));
                                                texcoord_index.push_back(absolute_index(c.texcoord, texcoord_count));
                                        }
                                        m.has_normal.push_back(normals ? 1 : 0);
                                        m.facet_material.push_back(material);
                                }
                                break;
                        }
                        case LineKind::USEMTL:
                        {
                                const Split s = split(lines.line(line));
                                const std::string name{read_name("material", s.rest_b, s.rest_e)};
                                const auto it = std::find(material_names.begin(), material_names.end(), name);
                                if (it != material_names.end())
                                {
                                        material = static_cast<int>(it - material_names.begin());
                                }
                                else
                                {
                                        material_names.push_back(name);
                                        m.material_colors.push_back({0.0f, 0.0f, 0.0f});
                                        material = static_cast<int>(material_names.size()) - 1;
                                        material_index.emplace(name, material);
                                }
                                break;
                        }
                        case LineKind::MTLLIB:
                        {
                                const Split s = split(lines.line(line));
                                const char* b = s.rest_b;
                                bool found = false;
                                while (true)
                                {
                                        while (b < s.rest_e && is_space(*b))
                                        {
                                                ++b;
                                        }
                                        if (b == s.rest_e)
                                        {
                                                break;
                                        }
                                        const char* e = b;
                                        while (e < s.rest_e && !is_space(*e))
                                        {
                                                ++e;
                                        }
                                        std::filesystem::path lib(std::string(b, e));
                                        found = true;
                                        if (unique_libraries.insert(lib).second)
                                        {
                                                libraries.push_back(lib);
                                        }
                                        b = e;
                                }
                                if (!found)
                                {
                                        fail("Line " + std::to_string(line) + ": mtllib " + std::string(s.rest_b, s.rest_e) +
                                             "\nLibrary name not found");
                                }
                                break;
                        }
                        }
                }
                if (!part.error.empty())
                {
                        fail(part.error);
                }
        }
        if (m.has_normal.empty())
        {
                fail("No facets found in OBJ file");
        }
        const int vertex_count = static_cast<int>(m.vertices.size() / n);
        const int normals_total = static_cast<int>(m.normals.size() / n);
        for (std::size_t f = 0; f < m.has_normal.size(); ++f)
        {
                for (int k = 0; k < n; ++k)
                {
                        const int v = m.facet_vertices[f * n + k];
                        if (v < 0 || v >= vertex_count)
                        {
                                fail("Vertex index " + std::to_string(v) + " is out of bounds [0, " +
                                     std::to_string(vertex_count) + ")");
                        }
                        const int t = texcoord_index[f * n + k];
                        if (t != -1 && (t < 0 || t >= texcoord_count))
                        {
                                fail("Texture coordinate index " + std::to_string(t) + " is out of bounds [0, " +
                                     std::to_string(texcoord_count) + ")");
                        }
                        const int nm = m.facet_normals[f * n + k];
                        if (m.has_normal[f] && (nm < 0 || nm >= normals_total))
                        {
                                fail("Normal index " + std::to_string(nm) + " is out of bounds [0, " +
                                     std::to_string(normals_total) + ")");
                        }
                }
        }

        // material libraries: Kd of every used material (obj/load_lib.cpp)
        const std::filesystem::path dir = path.parent_path();
        for (std::size_t l = 0; l < libraries.size() && !material_index.empty(); ++l)
        {
                const std::filesystem::path lib_name = dir / libraries[l];
                const Lines lib(read_bytes(lib_name));
                std::array<float, 3>* current = nullptr;
                for (std::size_t i = 0; i < lib.size(); ++i)
                {
                        const Split s = split(lib.line(i));
                        try
                        {
                                if (s.first == "newmtl")
                                {
                                        if (material_index.empty())
                                        {
                                                break;
                                        }
                                        const std::string name{read_name("material", s.rest_b, s.rest_e)};
                                        const auto it = material_index.find(name);
                                        if (it != material_index.end())
                                        {
                                                current = &m.material_colors[it->second];
                                                material_index.erase(it);
                                        }
                                        else
                                        {
                                                current = nullptr;
                                        }
                                }
                                else if (current && s.first == "Kd")
                                {
                                        read_color(s.rest_b, *current);
                                }
                                else if (current && s.first == "map_Kd")
                                {
                                        fail("Texture images are not supported");
                                }
                        }
                        catch (const std::exception& e)
                        {
                                fail("Library: " + lib_name.generic_string() + "\nLine " + std::to_string(i) + ": " +
                                     std::string(s.first) + " " + std::string(s.rest_b, s.rest_e) + "\n" + e.what());
                        }
                }
        }
        if (!material_index.empty())
        {
                std::string names;
                for (const auto& [name, index] : material_index)
                {
                        names += (names.empty() ? "" : ", ") + name;
                }
                fail("Materials not found in libraries: " + names);
        }
}

// ---------------------------------------------------------------------------
// STL (src/model/mesh/file/load_stl.cpp)

const char* skip(const char* p, const char* const last, bool (*pred)(char))
{
        while (p < last && pred(*p))
        {
                ++p;
        }
        return p;
}

bool not_new_line(const char c)
{
        return c != '\n';
}

const char* keyword(const char* p, const char* const last, const std::string_view word)
{
        if (p + word.size() > last || std::string_view(p, word.size()) != word)
        {
                fail("Keyword " + std::string(word) + " not found in STL file when expected");
        }
        const char* const q = p + word.size();
        if (q < last && !is_space(*q))
        {
                fail("Keyword " + std::string(word) + " not found in STL file when expected");
        }
        return q;
}

bool starts_with_keyword(const char* p, const char* const last, const std::string_view word)
{
        if (p + word.size() > last || std::string_view(p, word.size()) != word)
        {
                return false;
        }
        const char* const q = p + word.size();
        return !(q < last && !is_space(*q));
}

// vertices equal as float vectors (+0 equals -0, NaN equals nothing) share an index
class UniqueVertices final
{
        struct Key final
        {
                std::array<std::uint32_t, 5> bits{};

                bool operator==(const Key&) const = default;
        };

        struct Hash final
        {
                std::size_t operator()(const Key& k) const
                {
                        std::size_t h = 1469598103934665603ull;
                        for (const std::uint32_t b : k.bits)
                        {
                                h = (h ^ b) * 1099511628211ull;
                        }
                        return h;
                }
        };

        std::unordered_map<Key, int, Hash> map_;
        MeshFile& m_;

public:
        explicit UniqueVertices(MeshFile& m)
                : m_(m)
        {
        }

        int index(const float* v)
        {
                const int n = m_.n;
                Key key;
                bool nan = false;
                for (int i = 0; i < n; ++i)
                {
                        const float x = v[i] == 0.0f ? 0.0f : v[i];
                        nan = nan || x != x;
                        std::memcpy(&key.bits[i], &x, sizeof(float));
                }
                if (!nan)
                {
                        const auto it = map_.find(key);
                        if (it != map_.end())
                        {
                                return it->second;
                        }
                }
                const int index = static_cast<int>(m_.vertices.size() / n);
                m_.vertices.insert(m_.vertices.end(), v, v + n);
                if (!nan)
                {
                        map_.emplace(key, index);
                }
                return index;
        }
};

void add_stl_facet(MeshFile& m, UniqueVertices& unique, const float* vertices)
{
        for (int k = 0; k < m.n; ++k)
        {
                m.facet_vertices.push_back(unique.index(vertices + k * m.n));
                m.facet_normals.push_back(-1);
        }
        m.has_normal.push_back(0);
        m.facet_material.push_back(-1);
}

void read_stl(const std::filesystem::path& path, const int n, MeshFile& m)
{
        std::vector<char> data = read_bytes(path);
        UniqueVertices unique(m);
        const std::size_t header = 80;
        const std::size_t offset = header + sizeof(std::uint32_t);
        const std::size_t facet_bytes = static_cast<std::size_t>(n + n * n) * sizeof(float);
        bool binary = false;
        std::uint32_t count = 0;
        if (data.size() > offset)
        {
                std::memcpy(&count, &data[header], sizeof(count));
                const std::size_t required = offset + static_cast<std::size_t>(count) * facet_bytes;
                binary = data.size() >= required && data.size() <= required + sizeof(std::uint16_t) &&
                         std::any_of(data.begin(), data.end(),
                                     [](const char c)
                                     {
                                             return !is_print(c) && !is_space(c);
                                     });
        }
        if (binary)
        {
                std::vector<float> v(static_cast<std::size_t>(n) * n);
                const char* p = data.data() + offset + n * sizeof(float);
                for (std::uint32_t f = 0; f < count; ++f)
                {
                        std::memcpy(v.data(), p, v.size() * sizeof(float));
                        add_stl_facet(m, unique, v.data());
                        p += facet_bytes;
                }
        }
        else
        {
                data.push_back('\0');
                const char* p = data.data();
                const char* const last = data.data() + data.size() - 1;
                p = skip(p, last, is_space);
                p = keyword(p, last, "solid");
                p = skip(p, last, not_new_line);
                std::vector<float> v(static_cast<std::size_t>(n) * n);
                std::vector<float> normal(n);
                while (true)
                {
                        p = skip(p, last, is_space);
                        if (!starts_with_keyword(p, last, "facet normal"))
                        {
                                p = keyword(p, last, "endsolid");
                                p = skip(p, last, not_new_line);
                                p = skip(p, last, is_space);
                                if (p < last)
                                {
                                        fail("Nonspace found after solid end in STL file");
                                }
                                break;
                        }
                        p += std::string_view("facet normal").size();
                        if (p >= last)
                        {
                                fail("Normal coordinates not found in STL file when expected");
                        }
                        read_floats(p, normal.data(), n);
                        p = skip(p, last, is_space);
                        p = keyword(p, last, "outer loop");
                        for (int k = 0; k < n; ++k)
                        {
                                p = skip(p, last, is_space);
                                p = keyword(p, last, "vertex");
                                if (p >= last)
                                {
                                        fail("Vertex coordinates not found in STL file when expected");
                                }
                                read_floats(p, &v[static_cast<std::size_t>(k) * n], n);
                        }
                        p = skip(p, last, is_space);
                        p = keyword(p, last, "endloop");
                        p = skip(p, last, is_space);
                        p = keyword(p, last, "endfacet");
                        add_stl_facet(m, unique, v.data());
                }
        }
}

// mesh_facet.h: in 3-space facets whose edges are parallel are dropped
void remove_degenerate_facets(MeshFile& m)
{
        if (m.n != 3)
        {
                return;
        }
        const std::size_t count = m.has_normal.size();
        std::size_t out = 0;
        for (std::size_t f = 0; f < count; ++f)
        {
                const int* idx = &m.facet_vertices[f * 3];
                double e0[3];
                double e1[3];
                for (int d = 0; d < 3; ++d)
                {
                        const float a = m.vertices[idx[1] * 3 + d] - m.vertices[idx[0] * 3 + d];
                        const float b = m.vertices[idx[2] * 3 + d] - m.vertices[idx[0] * 3 + d];
                        e0[d] = a;
                        e1[d] = b;
                }
                const bool good = e0[1] * e1[2] - e0[2] * e1[1] != 0 || e0[0] * e1[2] - e0[2] * e1[0] != 0 ||
                                  e0[0] * e1[1] - e0[1] * e1[0] != 0;
                if (!good)
                {
                        continue;
                }
                if (out != f)
                {
                        for (int k = 0; k < 3; ++k)
                        {
                                m.facet_vertices[out * 3 + k] = m.facet_vertices[f * 3 + k];
                                m.facet_normals[out * 3 + k] = m.facet_normals[f * 3 + k];
                        }
                        m.has_normal[out] = m.has_normal[f];
                        m.facet_material[out] = m.facet_material[f];
                }
                ++out;
        }
        if (out == count)
        {
                return;
        }
        if (out == 0)
        {
                fail("No 2-facet found in 3-mesh");
        }
        m.facet_vertices.resize(out * 3);
        m.facet_normals.resize(out * 3);
        m.has_normal.resize(out);
        m.facet_material.resize(out);
}

std::string lower(std::string s)
{
        std::transform(s.begin(), s.end(), s.begin(),
                       [](const unsigned char c)
                       {
                               return static_cast<char>(std::tolower(c));
                       });
        return s;
}

// 1: OBJ, 2: STL; the dimension
std::array<int, 2> file_kind(const std::string& path)
{
        const std::string ext = lower(std::filesystem::path(path).extension().string());
        for (const auto& [name, kind] : {std::pair<std::string_view, int>{".obj", 1}, {".stl", 2}})
        {
                if (ext.size() < name.size() || std::string_view(ext).substr(0, name.size()) != name)
                {
                        continue;
                }
                const std::string_view digits = std::string_view(ext).substr(name.size());
                if (digits.empty())
                {
                        return {kind, 3};
                }
                int n = 0;
                const auto [ptr, ec] = std::from_chars(digits.data(), digits.data() + digits.size(), n);
                if (ec == std::errc{} && ptr == digits.data() + digits.size() && n >= 3)
                {
                        return {kind, n};
                }
        }
        return {0, 0};
}
} // namespace

int mesh_file_dimension(const std::string& path)
{
        return file_kind(path)[1];
}

MeshFile load_mesh_file(const std::string& path, const int n)
{
        const auto [kind, dimension] = file_kind(path);
        if (kind == 0)
        {
                fail("Not an OBJ or STL file name: " + path);
        }
        if (dimension != n)
        {
                fail("Requested file dimension " + std::to_string(n) + ", detected file dimension " +
                     std::to_string(dimension) + ", file " + path);
        }
        MeshFile m;
        m.n = n;
        if (kind == 1)
        {
                read_obj(path, n, m);
        }
        else
        {
                read_stl(path, n, m);
        }
        remove_degenerate_facets(m);
        return m;
}
} // namespace nbpt::host
