// ats_io.cpp -- on-disk formats (host only).
//
//   OBJ export of positions and triangles, as SimMesh::saveToOBJ_combined /
//   SolverInterface::save_mesh_to_obj write it (src/Utils/mesh_reader.cpp:374-462,
//   examples/example2_async_iter.cpp:1649-1710): "v x y z" lines, 1-based "f a b c".
//   Binary cloth state (x, v) for checkpoint / resume and trajectories, a versioned
//   little-endian layout (the reference's save_to_binary, mesh_reader.h:323-343, dumps
//   raw arrays with no header):
//     offset 0  char[4]  "ATSS"
//            4  u32      version (1)
//            8  u32      vertex count n
//           12  u32      frame index
//           16  f32[3n]  positions
//              f32[3n]  velocities
//              u64      FNV-1a 64 of every byte from offset 0 up to here

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ats_cloth.h"

namespace ats {
void set_error(const std::string& msg);
}

namespace {

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

bool little_endian() {
    const uint32_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

}  // namespace

extern "C" {

int ats_obj_write(const char* path, const float* positions, int num_verts, const int* faces, int num_faces) {
    if (!path || !positions || num_verts <= 0 || num_faces < 0 || (num_faces > 0 && !faces)) {
        ats::set_error("ats_obj_write: bad arguments");
        return ATS_ERR_INVALID;
    }
    FILE* f = std::fopen(path, "w");
    if (!f) {
        ats::set_error(std::string("ats_obj_write: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    std::fprintf(f, "o mesh_0\n");
    for (int i = 0; i < num_verts; ++i)
        std::fprintf(f, "v %.9g %.9g %.9g\n", positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    for (int i = 0; i < num_faces; ++i)
        std::fprintf(f, "f %d %d %d\n", faces[3 * i] + 1, faces[3 * i + 1] + 1, faces[3 * i + 2] + 1);
    const bool ok = std::fclose(f) == 0;
    if (!ok) {
        ats::set_error("ats_obj_write: write failed");
        return ATS_ERR_INVALID;
    }
    return ATS_OK;
}

int ats_state_write(const char* path, const float* x, const float* v, int num_verts, int frame) {
    if (!path || !x || !v || num_verts <= 0 || frame < 0) {
        ats::set_error("ats_state_write: bad arguments");
        return ATS_ERR_INVALID;
    }
    if (!little_endian()) {
        ats::set_error("ats_state_write: big-endian hosts are not supported");
        return ATS_ERR_INVALID;
    }
    const size_t n3 = 3 * (size_t)num_verts;
    std::vector<unsigned char> buf(16 + 8 * n3);
    std::memcpy(buf.data(), "ATSS", 4);
    const uint32_t hdr[3] = {1u, (uint32_t)num_verts, (uint32_t)frame};
    std::memcpy(buf.data() + 4, hdr, 12);
    std::memcpy(buf.data() + 16, x, 4 * n3);
    std::memcpy(buf.data() + 16 + 4 * n3, v, 4 * n3);
    const uint64_t sum = fnv1a(buf.data(), buf.size());
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        ats::set_error(std::string("ats_state_write: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size() && std::fwrite(&sum, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        ats::set_error("ats_state_write: write failed");
        return ATS_ERR_INVALID;
    }
    return ATS_OK;
}

int ats_state_read(const char* path, float* x, float* v, int* num_verts, int* frame) {
    if (!path || !num_verts) {
        ats::set_error("ats_state_read: bad arguments");
        return ATS_ERR_INVALID;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        ats::set_error(std::string("ats_state_read: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    unsigned char head[16];
    if (std::fread(head, 1, 16, f) != 16 || std::memcmp(head, "ATSS", 4) != 0) {
        std::fclose(f);
        ats::set_error("ats_state_read: not a cloth state file");
        return ATS_ERR_INVALID;
    }
    uint32_t hdr[3];
    std::memcpy(hdr, head + 4, 12);
    if (hdr[0] != 1u) {
        std::fclose(f);
        ats::set_error("ats_state_read: unsupported version " + std::to_string(hdr[0]));
        return ATS_ERR_INVALID;
    }
    const int n = (int)hdr[1];
    if (!x || !v) {  // size query
        std::fclose(f);
        *num_verts = n;
        if (frame) *frame = (int)hdr[2];
        return ATS_OK;
    }
    if (*num_verts < n) {
        std::fclose(f);
        ats::set_error("ats_state_read: output arrays too small");
        return ATS_ERR_INVALID;
    }
    const size_t n3 = 3 * (size_t)n;
    std::vector<unsigned char> buf(16 + 8 * n3);
    std::memcpy(buf.data(), head, 16);
    uint64_t sum = 0;
    const bool ok = std::fread(buf.data() + 16, 1, 8 * n3, f) == 8 * n3 && std::fread(&sum, 8, 1, f) == 1;
    std::fclose(f);
    if (!ok) {
        ats::set_error("ats_state_read: file is truncated");
        return ATS_ERR_INVALID;
    }
    if (fnv1a(buf.data(), buf.size()) != sum) {
        ats::set_error("ats_state_read: checksum mismatch");
        return ATS_ERR_INVALID;
    }
    std::memcpy(x, buf.data() + 16, 4 * n3);
    std::memcpy(v, buf.data() + 16 + 4 * n3, 4 * n3);
    *num_verts = n;
    if (frame) *frame = (int)hdr[2];
    return ATS_OK;
}

}  // extern "C"
