// sceneio.cu -- mesh files in, for scenes the caller does not generate.
//
// The reference's Scene loads each frame of a benchmark from a file
// (Scene::update / addMesh, Mine/world/Scene.cpp:14-43, through assimp with
// aiProcess_Triangulate, Mine/utility/ModelReader.hpp:23-27; the file of
// frame f is a printf pattern, CDBenchmarkSettings::file_name,
// Mine/setting/CDBenchmarkSettings.h:36-43) and concatenates the meshes of a
// file, offsetting vertex ids.  This reads Wavefront OBJ, the format of the
// reference's benchmark sequences, with no library: vertex records (v x y z)
// and face records (f with v, v/vt, v//vn or v/vt/vn corners, negative ids
// relative to the vertices read so far); polygons are split into a fan of
// triangles around their first corner; other records (vt, vn, o, g, s,
// usemtl, mtllib, comments) are skipped.  Vertex ids stay as the file shares
// them, so adjacent triangles keep their common vertices (assimp's OBJ import
// gives every face corner a vertex of its own).
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/bvhcd.h"

namespace {

struct ObjData {
    std::vector<float> pos;
    std::vector<int32_t> faces;
};

// parses one face corner ("12", "12/3", "12//5", "-1/2/3"); returns the
// 0-based vertex id or -1 on a malformed or out-of-range id
long corner(const char *tok, long nverts) {
    char *end = nullptr;
    errno = 0;
    long id = std::strtol(tok, &end, 10);
    if (end == tok || errno) return -1;
    if (*end != '\0' && *end != '/') return -1;
    if (id > 0) id -= 1;
    else if (id < 0) id += nverts;
    else return -1;
    return (id >= 0 && id < nverts) ? id : -1;
}

bvhcd_status read_obj(const char *path, ObjData &d) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return BVHCD_INVALID_ARG;
    char *buf = nullptr;
    size_t cap = 0;
    std::vector<long> poly;
    bvhcd_status st = BVHCD_OK;
    while (getline(&buf, &cap, f) >= 0) {
        char *s = buf;
        while (*s == ' ' || *s == '\t') ++s;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            float x, y, z;
            if (std::sscanf(s + 2, "%f %f %f", &x, &y, &z) != 3) { st = BVHCD_INVALID_ARG; break; }
            d.pos.push_back(x);
            d.pos.push_back(y);
            d.pos.push_back(z);
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            poly.clear();
            const long nv = (long)(d.pos.size() / 3);
            char *save = nullptr;
            for (char *tok = strtok_r(s + 2, " \t\r\n", &save); tok; tok = strtok_r(nullptr, " \t\r\n", &save)) {
                const long id = corner(tok, nv);
                if (id < 0) { st = BVHCD_INVALID_ARG; break; }
                poly.push_back(id);
            }
            if (st != BVHCD_OK) break;
            if (poly.size() < 3) { st = BVHCD_INVALID_ARG; break; }
            for (size_t k = 1; k + 1 < poly.size(); k++) {
                d.faces.push_back((int32_t)poly[0]);
                d.faces.push_back((int32_t)poly[k]);
                d.faces.push_back((int32_t)poly[k + 1]);
            }
        }
        if (d.pos.size() / 3 > 0x7fffffffu || d.faces.size() / 3 > 0x7fffffffu) { st = BVHCD_INVALID_ARG; break; }
    }
    if (st == BVHCD_OK && std::ferror(f)) st = BVHCD_INVALID_ARG;
    std::free(buf);
    std::fclose(f);
    return st;
}

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

bvhcd_status bvhcd_obj_read(const char *path, float *pos, int32_t vcap, int32_t *faces, int32_t fcap,
                            int32_t *num_vertices, int32_t *num_faces) {
    if (!path || vcap < 0 || fcap < 0) return BVHCD_INVALID_ARG;
    ObjData d;
    bvhcd_status st = read_obj(path, d);
    if (st != BVHCD_OK) return st;
    const int32_t V = (int32_t)(d.pos.size() / 3), T = (int32_t)(d.faces.size() / 3);
    if (num_vertices) *num_vertices = V;
    if (num_faces) *num_faces = T;
    if (pos) std::memcpy(pos, d.pos.data(), sizeof(float) * 3 * (size_t)(V < vcap ? V : vcap));
    if (faces) std::memcpy(faces, d.faces.data(), sizeof(int32_t) * 3 * (size_t)(T < fcap ? T : fcap));
    if ((pos && V > vcap) || (faces && T > fcap)) return BVHCD_CAPACITY_EXCEEDED;
    return BVHCD_OK;
}

#pragma GCC visibility pop
}
