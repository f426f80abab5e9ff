// Mesh files: OBJ (n = 3) and OBJ-n (.objN, n > 3), read as the reference's loader reads their
// geometry (src/obj/file/file_load.cpp): "v" lines of n coordinates, "vn" lines of n normal
// components, "f" lines of vertex[/texture[/normal]] index groups (1-based; negative: counted back
// from the last element read so far), a facet of more than n groups split into a fan around its first
// group (read_facets, file_load.cpp:406-445).  Texture coordinates, materials, groups and every other
// line are not used by the painter's geometry and are skipped.
#include "ntrace.h"

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace ntrace
{
int report_error(int code, const std::string& message);
}

namespace
{
struct Parsed
{
        std::vector<float> vertices;
        std::vector<float> normals;
        std::vector<int32_t> facets;
        std::vector<int32_t> facet_normals;  // -1: the facet has no normals
        long long facets_with_normals = 0;
};

bool is_space(char c)
{
        return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// one index of a group: returns false on a syntax error; *value 0 when absent
bool read_index(const char*& p, const char* end, long* value)
{
        if (p == end || is_space(*p) || *p == '/')
        {
                *value = 0;
                return true;
        }
        char* q = nullptr;
        errno = 0;
        long v = std::strtol(p, &q, 10);
        if (q == p || errno)
        {
                return false;
        }
        p = q;
        *value = v;
        return true;
}

int parse(const char* path, int n, Parsed* out, std::string* err)
{
        FILE* f = std::fopen(path, "rb");
        if (!f)
        {
                *err = std::string("cannot open ") + path;
                return NT_EINVAL;
        }
        std::string line;
        std::vector<char> buf(1 << 16);
        long long line_no = 0;
        auto fail = [&](const std::string& m) {
                *err = std::string(path) + ":" + std::to_string(line_no) + ": " + m;
                return NT_EINVAL;
        };
        int rc = NT_OK;
        while (rc == NT_OK)
        {
                line.clear();
                bool got = false;
                while (std::fgets(buf.data(), (int)buf.size(), f))
                {
                        got = true;
                        line += buf.data();
                        if (!line.empty() && line.back() == '\n')
                        {
                                break;
                        }
                }
                if (!got)
                {
                        break;
                }
                ++line_no;
                const char* p = line.c_str();
                const char* end = p + line.size();
                while (p < end && is_space(*p))
                {
                        ++p;
                }
                const char* key = p;
                while (p < end && !is_space(*p))
                {
                        ++p;
                }
                const std::string k(key, p);
                if (k == "v" || k == "vn")
                {
                        std::vector<float>& dst = (k == "v") ? out->vertices : out->normals;
                        for (int i = 0; i < n; ++i)
                        {
                                char* q = nullptr;
                                float x = std::strtof(p, &q);
                                if (q == p)
                                {
                                        rc = fail("expected " + std::to_string(n) + " numbers after " + k);
                                        break;
                                }
                                p = q;
                                dst.push_back(x);
                        }
                }
                else if (k == "f")
                {
                        std::vector<long> gv, gn;
                        while (true)
                        {
                                while (p < end && is_space(*p))
                                {
                                        ++p;
                                }
                                if (p >= end)
                                {
                                        break;
                                }
                                long v = 0, t = 0, nn = 0;
                                if (!read_index(p, end, &v) || v == 0)
                                {
                                        rc = fail("bad facet vertex index");
                                        break;
                                }
                                if (p < end && *p == '/')
                                {
                                        ++p;
                                        if (!read_index(p, end, &t))
                                        {
                                                rc = fail("bad facet texture index");
                                                break;
                                        }
                                        if (p < end && *p == '/')
                                        {
                                                ++p;
                                                if (!read_index(p, end, &nn))
                                                {
                                                        rc = fail("bad facet normal index");
                                                        break;
                                                }
                                        }
                                }
                                if (p < end && !is_space(*p))
                                {
                                        rc = fail("bad facet group");
                                        break;
                                }
                                gv.push_back(v);
                                gn.push_back(nn);
                        }
                        if (rc != NT_OK)
                        {
                                break;
                        }
                        if ((int)gv.size() < n)
                        {
                                rc = fail("facet with " + std::to_string(gv.size()) + " vertices (min = " + std::to_string(n) + ")");
                                break;
                        }
                        int with_normals = 0;
                        for (long x : gn)
                        {
                                with_normals += x != 0;
                        }
                        if (!(with_normals == 0 || with_normals == (int)gn.size()))
                        {
                                rc = fail("inconsistent facet normal indices");
                                break;
                        }
                        const long nv = (long)(out->vertices.size() / n);
                        const long nnorm = (long)(out->normals.size() / n);
                        auto vidx = [&](long v) { return v > 0 ? v - 1 : nv + v; };
                        auto nidx = [&](long x) { return x > 0 ? x - 1 : (x < 0 ? nnorm + x : -1); };
                        // a fan around the first group (read_facets, file_load.cpp:428-444)
                        const int count = (int)gv.size() - (n - 1);
                        for (int i = 0; i < count; ++i)
                        {
                                for (int j = 0; j < n; ++j)
                                {
                                        const int g = (j == 0) ? 0 : i + j;
                                        const long vi = vidx(gv[g]);
                                        const long ni = nidx(gn[g]);
                                        if (vi < 0 || vi >= nv || (with_normals && (ni < 0 || ni >= nnorm)))
                                        {
                                                rc = fail("facet index out of range");
                                                break;
                                        }
                                        out->facets.push_back((int32_t)vi);
                                        out->facet_normals.push_back(with_normals ? (int32_t)ni : -1);
                                }
                                if (rc != NT_OK)
                                {
                                        break;
                                }
                                out->facets_with_normals += with_normals ? 1 : 0;
                        }
                }
        }
        std::fclose(f);
        if (rc == NT_OK && out->facets.empty())
        {
                *err = std::string("no facets found in ") + path;
                rc = NT_EINVAL;
        }
        return rc;
}
}

extern "C" int nt_scene_add_obj_file(nt_scene* scene, const char* path, const nt_surface* surface)
{
        if (!scene || !path)
        {
                return ntrace::report_error(NT_EINVAL, "null argument");
        }
        const int n = nt_scene_dimension(scene);
        if (n < 3)
        {
                return ntrace::report_error(NT_EINVAL, "bad scene");
        }
        Parsed m;
        std::string err;
        int rc = parse(path, n, &m, &err);
        if (rc != NT_OK)
        {
                return ntrace::report_error(rc, err);
        }
        const int64_t nv = (int64_t)(m.vertices.size() / n);
        const int64_t nf = (int64_t)(m.facets.size() / n);
        rc = nt_scene_add_mesh(scene, m.vertices.data(), nv, m.facets.data(), nf, surface);
        if (rc != NT_OK || m.facets_with_normals == 0)
        {
                return rc;
        }
        // the mesh just added is the last object
        return nt_scene_set_mesh_normals(scene, nt_scene_object_count(scene) - 1, m.normals.data(),
                                         (int64_t)(m.normals.size() / n), m.facet_normals.data());
}
