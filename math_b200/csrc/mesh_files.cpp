#include "mesh_files.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

namespace nbpt::host
{
namespace
{
[[noreturn]] void fail(const std::string& message)
{
        throw std::runtime_error(message);
}

// Host threads for `count` items of work in parts of at least `grain`.
unsigned part_count(const std::size_t count, const std::size_t grain)
{
        const std::size_t threads = std::max(1u, std::thread::hardware_concurrency());
        return static_cast<unsigned>(std::max<std::size_t>(1, std::min(threads, count / grain)));
}

// fn(part, begin, end) over `parts` consecutive ranges of [0, count), part 0
// on the calling thread; fn must not throw.
template <typename F>
void parallel_parts(const std::size_t count, const unsigned parts, const F& fn)
{
        const std::size_t step = (count + parts - 1) / parts;
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < parts; ++t)
        {
                pool.emplace_back(
                        [&, t]
                        {
                                fn(t, std::min(count, t * step), std::min(count, (t + 1) * step));
                        });
        }
        fn(0u, std::size_t{0}, std::min(count, step));
        for (std::thread& th : pool)
        {
                th.join();
        }
}

// A file's bytes, with room for one byte more (a line end or a terminator).
struct Bytes final
{
        std::unique_ptr<char[]> buffer;
        std::size_t size = 0;

        char* data()
        {
                return buffer.get();
        }

        const char* data() const
        {
                return buffer.get();
        }
};

// The file read in parts by the host threads into an uninitialised buffer,
// so that the buffer's pages are first touched by the readers in parallel.
Bytes read_bytes(const std::filesystem::path& path)
{
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0)
        {
                fail("Failed to open file " + path.generic_string());
        }
        struct stat st;
        if (::fstat(fd, &st) != 0)
        {
                ::close(fd);
                fail("Failed to read file " + path.generic_string());
        }
        Bytes bytes;
        bytes.size = static_cast<std::size_t>(st.st_size);
        bytes.buffer.reset(new char[bytes.size + 1]);
        std::atomic<bool> ok{true};
        parallel_parts(bytes.size, part_count(bytes.size, std::size_t{1} << 22),
                       [&](unsigned, const std::size_t b, const std::size_t e)
                       {
                               std::size_t done = b;
                               while (done < e)
                               {
                                       const ssize_t r = ::pread(fd, bytes.data() + done, e - done, static_cast<off_t>(done));
                                       if (r <= 0)
                                       {
                                               ok = false;
                                               return;
                                       }
                                       done += static_cast<std::size_t>(r);
                               }
                       });
        ::close(fd);
        if (!ok)
        {
                fail("Failed to read file " + path.generic_string());
        }
        return bytes;
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

// ASCII letters and digits (std::isalnum of the C locale, without its call)
// and the other characters strtof's forms use: . + - ( ) _
bool number_char(const char c)
{
        const char lower = static_cast<char>(c | 0x20);
        return (c >= '0' && c <= '9') || (lower >= 'a' && lower <= 'z') || c == '.' || c == '+' || c == '-' ||
               c == '(' || c == ')' || c == '_';
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
        while (number_char(*line_end))
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
        Bytes data;
        std::vector<std::size_t> begin; // each line's start, then the end of the text

        explicit Lines(Bytes&& text)
                : data(std::move(text))
        {
                if (data.size == 0)
                {
                        return;
                }
                if (data.data()[data.size - 1] != '\n')
                {
                        data.data()[data.size++] = '\n';
                }
                if (std::memchr(data.data(), '\0', data.size) != nullptr)
                {
                        fail("Text data contains null character");
                }
                // the line ends found in parts on the host threads, then
                // joined in order
                const unsigned parts = part_count(data.size, std::size_t{1} << 20);
                std::vector<std::vector<std::size_t>> ends(parts);
                parallel_parts(data.size, parts,
                               [&](const unsigned t, const std::size_t b, const std::size_t e)
                               {
                                       char* p = data.data() + b;
                                       char* const last = data.data() + e;
                                       while (p < last)
                                       {
                                               p = static_cast<char*>(std::memchr(p, '\n', last - p));
                                               if (p == nullptr)
                                               {
                                                       break;
                                               }
                                               ends[t].push_back(p - data.data());
                                               *p++ = '\0';
                                       }
                               });
                std::size_t lines = 0;
                for (const std::vector<std::size_t>& part : ends)
                {
                        lines += part.size();
                }
                begin.reserve(lines + 1);
                begin.push_back(0);
                for (const std::vector<std::size_t>& part : ends)
                {
                        for (const std::size_t end : part)
                        {
                                begin.push_back(end + 1);
                        }
                }
        }

        std::size_t size() const
        {
                return begin.empty() ? 0 : begin.size() - 1;
        }

        // the line without its terminator
        std::string_view line(const std::size_t i) const
        {
                return {data.data() + begin[i], begin[i + 1] - begin[i] - 1};
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
        const void* const comment = std::memchr(q, '#', last - q);
        const char* const e = comment != nullptr ? static_cast<const char*>(comment) : last;
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
        int material = -1;
        std::map<std::string, int, std::less<>> material_index; // materials still to find in the libraries
        std::vector<std::string> material_names;
        std::vector<std::filesystem::path> libraries;
        std::set<std::filesystem::path> unique_libraries;

        const Lines lines(read_bytes(path));

        // parse the lines in parts on the host threads, then apply them in order
        const std::size_t line_count = lines.size();
        const unsigned threads = part_count(line_count, 4096);
        std::vector<ObjPart> parts(threads);
        parallel_parts(line_count, threads,
                       [&](const unsigned t, const std::size_t b, const std::size_t e)
                       {
                               parse_obj_lines(lines, b, e, n, max_corners, parts[t]);
                       });

        // In order over the parts: the running counts where each part starts
        // and its facets' place, and the usemtl and mtllib lines, whose
        // failures, like a part's parse error, come after the lines before
        // them are taken.
        struct PartStart final
        {
                std::size_t vertices = 0;
                std::size_t normals = 0;
                std::size_t texcoords = 0;
                std::size_t facets = 0;
                int material = -1;
                std::vector<int> materials; // the material of each usemtl line of the part
        };
        std::vector<PartStart> starts(parts.size());
        std::size_t vertices = 0;
        std::size_t normals = 0;
        std::size_t texcoords = 0;
        std::size_t facets = 0;
        std::size_t i = 0;
        for (std::size_t p = 0; p < parts.size(); ++p)
        {
                const ObjPart& part = parts[p];
                PartStart& start = starts[p];
                start.vertices = vertices;
                start.normals = normals;
                start.texcoords = texcoords;
                start.facets = facets;
                start.material = material;
                std::size_t facet_line = 0;
                for (const LineKind kind : part.kind)
                {
                        const std::size_t line = i++;
                        switch (kind)
                        {
                        case LineKind::NONE:
                                break;
                        case LineKind::V:
                                ++vertices;
                                break;
                        case LineKind::VT:
                                ++texcoords;
                                break;
                        case LineKind::VN:
                                ++normals;
                                break;
                        case LineKind::F:
                                // a fan around the first corner
                                facets += part.corner_count[facet_line++] - n + 1;
                                break;
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
                                start.materials.push_back(material);
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
        texcoord_count = static_cast<int>(texcoords);

        // the parts' vertices, normals and facets written in parallel
        m.vertices.resize(vertices * n);
        m.normals.resize(normals * n);
        m.facet_vertices.resize(facets * n);
        m.facet_normals.resize(facets * n);
        texcoord_index.resize(facets * n);
        m.has_normal.resize(facets);
        m.facet_material.resize(facets);
        parallel_parts(
                parts.size(), static_cast<unsigned>(parts.size()),
                [&](unsigned, const std::size_t part_begin, const std::size_t part_end)
                {
                        for (std::size_t p = part_begin; p < part_end; ++p)
                        {
                                const ObjPart& part = parts[p];
                                const PartStart& start = starts[p];
                                std::size_t v = start.vertices;
                                std::size_t vn = start.normals;
                                std::size_t vt = start.texcoords;
                                std::size_t f = start.facets;
                                int facet_material = start.material;
                                std::size_t usemtl = 0;
                                std::size_t value = 0;
                                std::size_t facet_line = 0;
                                std::size_t corner = 0;
                                for (const LineKind kind : part.kind)
                                {
                                        switch (kind)
                                        {
                                        case LineKind::V:
                                                std::copy_n(part.values.begin() + value, n, m.vertices.begin() + v * n);
                                                value += n;
                                                ++v;
                                                break;
                                        case LineKind::VT:
                                                ++vt;
                                                break;
                                        case LineKind::VN:
                                                std::copy_n(part.values.begin() + value, n, m.normals.begin() + vn * n);
                                                value += n;
                                                ++vn;
                                                break;
                                        case LineKind::F:
                                        {
                                                const int count = part.corner_count[facet_line++];
                                                const Corner* const c0 = &part.corners[corner];
                                                corner += count;
                                                const int vertex_count = static_cast<int>(v);
                                                const bool with_normals = c0[0].normal != 0;
                                                for (int fan = 0; fan + n - 1 < count; ++fan, ++f)
                                                {
                                                        for (int k = 0; k < n; ++k)
                                                        {
                                                                const Corner& c = c0[k == 0 ? 0 : fan + k];
                                                                m.facet_vertices[f * n + k] =
                                                                        c.vertex > 0 ? c.vertex - 1 : vertex_count + c.vertex;
                                                                m.facet_normals[f * n + k] =
                                                                        absolute_index(c.normal, static_cast<int>(vn));
                                                                texcoord_index[f * n + k] =
                                                                        absolute_index(c.texcoord, static_cast<int>(vt));
                                                        }
                                                        m.has_normal[f] = with_normals ? 1 : 0;
                                                        m.facet_material[f] = facet_material;
                                                }
                                                break;
                                        }
                                        case LineKind::USEMTL:
                                                facet_material = start.materials[usemtl++];
                                                break;
                                        case LineKind::NONE:
                                        case LineKind::MTLLIB:
                                                break;
                                        }
                                }
                        }
                });
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

// A corner's coordinates as a map key: the float bits with -0 as +0.
struct VertexKey final
{
        std::array<std::uint32_t, 5> bits{};

        bool operator==(const VertexKey&) const = default;
};

struct VertexKeyHash final
{
        std::size_t operator()(const VertexKey& k) const
        {
                std::size_t h = 1469598103934665603ull;
                for (const std::uint32_t b : k.bits)
                {
                        h = (h ^ b) * 1099511628211ull;
                }
                return h;
        }
};

// false for a corner with a NaN coordinate
bool vertex_key(const float* const v, const int n, VertexKey& key)
{
        for (int i = 0; i < n; ++i)
        {
                const float x = v[i] == 0.0f ? 0.0f : v[i];
                if (x != x)
                {
                        return false;
                }
                std::memcpy(&key.bits[i], &x, sizeof(float));
        }
        return true;
}

// The STL facets from their corners: facet f's n corners of n floats start
// at base + f * stride.  Corners equal as float vectors (+0 equals -0, NaN
// equals nothing) share one vertex, and the vertices are numbered in order
// of first appearance, as one map filled corner by corner numbers them.  The
// corners are hashed into one group per host thread; each thread fills its
// group's map in corner order, so it meets each of its vertices first where
// the vertex first appears, and the numbering is a running count of first
// appearances over all corners.  The per-corner scratch is left
// uninitialised, so that its pages are first touched by the threads.
void add_stl_facets(MeshFile& m, const char* const base, const std::size_t stride, const std::size_t facets)
{
        const int n = m.n;
        const std::size_t count = facets * n;
        const auto corner = [&](const std::size_t c, float* const v)
        {
                std::memcpy(v, base + (c / n) * stride + (c % n) * n * sizeof(float), n * sizeof(float));
        };
        constexpr std::uint32_t NO_GROUP = 0xffffffffu;
        const unsigned groups = part_count(count, std::size_t{1} << 15);

        const std::unique_ptr<std::uint32_t[]> group(new std::uint32_t[count]);
        const std::unique_ptr<std::size_t[]> first(new std::size_t[count]); // where the vertex first appears
        parallel_parts(count, groups,
                       [&](unsigned, const std::size_t b, const std::size_t e)
                       {
                               float v[5];
                               for (std::size_t c = b; c < e; ++c)
                               {
                                       corner(c, v);
                                       VertexKey key;
                                       if (vertex_key(v, n, key))
                                       {
                                               group[c] = static_cast<std::uint32_t>(VertexKeyHash()(key) % groups);
                                       }
                                       else
                                       {
                                               group[c] = NO_GROUP;
                                       }
                                       first[c] = c;
                               }
                       });
        parallel_parts(groups, groups,
                       [&](const unsigned t, std::size_t, std::size_t)
                       {
                               std::unordered_map<VertexKey, std::size_t, VertexKeyHash> map;
                               float v[5];
                               for (std::size_t c = 0; c < count; ++c)
                               {
                                       if (group[c] != t)
                                       {
                                               continue;
                                       }
                                       corner(c, v);
                                       VertexKey key;
                                       vertex_key(v, n, key);
                                       first[c] = map.try_emplace(key, c).first->second;
                               }
                       });

        // vertex numbers at first appearances (in the group array, no longer
        // needed), then every corner's vertex and the vertices' coordinates
        std::uint32_t* const number = group.get();
        std::uint32_t vertices = 0;
        for (std::size_t c = 0; c < count; ++c)
        {
                if (first[c] == c)
                {
                        number[c] = vertices++;
                }
        }
        m.vertices.resize(static_cast<std::size_t>(vertices) * n);
        m.facet_vertices.resize(count);
        parallel_parts(count, groups,
                       [&](unsigned, const std::size_t b, const std::size_t e)
                       {
                               for (std::size_t c = b; c < e; ++c)
                               {
                                       const std::uint32_t v = number[first[c]];
                                       m.facet_vertices[c] = static_cast<int>(v);
                                       if (first[c] == c)
                                       {
                                               corner(c, &m.vertices[static_cast<std::size_t>(v) * n]);
                                       }
                               }
                       });
        m.facet_normals.assign(count, -1);
        m.has_normal.assign(facets, 0);
        m.facet_material.assign(facets, -1);
}

void read_stl(const std::filesystem::path& path, const int n, MeshFile& m)
{
        Bytes data = read_bytes(path);
        const std::size_t header = 80;
        const std::size_t offset = header + sizeof(std::uint32_t);
        const std::size_t facet_bytes = static_cast<std::size_t>(n + n * n) * sizeof(float);
        bool binary = false;
        std::uint32_t count = 0;
        if (data.size > offset)
        {
                std::memcpy(&count, data.data() + header, sizeof(count));
                const std::size_t required = offset + static_cast<std::size_t>(count) * facet_bytes;
                binary = data.size >= required && data.size <= required + sizeof(std::uint16_t) &&
                         std::any_of(data.data(), data.data() + data.size,
                                     [](const char c)
                                     {
                                             return !is_print(c) && !is_space(c);
                                     });
        }
        if (binary)
        {
                // per facet: n normal floats (unused), then n corners of n floats
                add_stl_facets(m, data.data() + offset + n * sizeof(float), facet_bytes, count);
        }
        else
        {
                std::vector<float> corners; // each facet's n corners
                data.data()[data.size] = '\0';
                const char* p = data.data();
                const char* const last = data.data() + data.size;
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
                        corners.insert(corners.end(), v.begin(), v.end());
                }
                const std::size_t facet_floats = static_cast<std::size_t>(n) * n;
                add_stl_facets(m, reinterpret_cast<const char*>(corners.data()), facet_floats * sizeof(float),
                               corners.size() / facet_floats);
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
