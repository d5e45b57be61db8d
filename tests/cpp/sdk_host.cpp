// A C++ host driving libvision_b200 the way the reference's SDK user drives
// vision-renderer.dll (src/sdk/vision.h:66-80): scene from JSON, geometry
// added through add_instance, build_accel, camera, render, download.  Built
// and run by tests/test_sdk.py against include/vision_b200.h, so the header
// and the library's exports cannot drift apart unnoticed.
//
// usage: sdk_host <scene.json> <device: -1 host only | 0..> <frames> [film.bin]
// Prints "prims=<n> instances=<n> lights=<n>" and, with a device, writes the
// linear film (float4 per pixel) to film.bin.
#include "vision_b200.h"

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

static std::string read_file(const char *path) {
    std::ifstream in(path, std::ios::binary);
    std::stringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s scene.json device frames [film.bin]\n", argv[0]);
        return 2;
    }
    const int device = std::atoi(argv[2]);
    const uint32_t frames = static_cast<uint32_t>(std::atoi(argv[3]));
    vs_context *ctx = nullptr;
    if (vs_context_create(device, &ctx) != VS_OK) {
        std::fprintf(stderr, "no context on device %d\n", device);
        return 3;
    }
    std::string json = read_file(argv[1]);
    vs_scene *scene = nullptr;
    if (vs_scene_load_json(ctx, json.data(), json.size(), ".", nullptr, &scene) != VS_OK) {
        std::fprintf(stderr, "load: %s\n", vs_last_error(ctx));
        return 4;
    }
    // A 0.3 x 0.3 x 0.3 box as an SDK instance: 8 corners, 12 triangles
    // (outward winding), rotated -18 degrees about y and placed on the floor.
    const float h = 0.15f;
    std::vector<vs_vertex> v(8);
    for (int i = 0; i < 8; ++i) {
        v[i] = vs_vertex{{(i & 1) ? h : -h, (i & 2) ? h : -h, (i & 4) ? h : -h}, {0, 0, 0}, {0, 0}, {0, 0}};
    }
    const uint32_t tri[36] = {0, 2, 1, 1, 2, 3, 4, 5, 6, 5, 7, 6, 0, 1, 4, 1, 5, 4,
                              2, 6, 3, 3, 6, 7, 0, 4, 2, 2, 4, 6, 1, 3, 5, 3, 7, 5};
    const float c = 0.95105652f, s = -0.30901699f;  // cos, sin of -18 degrees
    const float o2w[16] = {c, 0, -s, 0, 0, 1, 0, 0, s, 0, c, 0, 0.17f, 0.15f, 0.12f, 1};  // column-major
    uint32_t inst = 0;
    if (vs_scene_add_instance(scene, v.data(), 8, tri, 12, o2w, "{\"type\": \"diffuse\", \"param\": {\"color\": [0.2, 0.6, 0.3]}}",
                              &inst) != VS_OK) {
        std::fprintf(stderr, "add_instance: %s\n", vs_last_error(ctx));
        return 5;
    }
    if (vs_scene_build_accel(scene) != VS_OK) {
        std::fprintf(stderr, "build_accel: %s\n", vs_last_error(ctx));
        return 6;
    }
    vs_scene_info info{};
    vs_scene_info_get(scene, &info);
    std::printf("prims=%u instances=%u lights=%u added=%u\n", info.prim_count, info.instance_count, info.light_count,
                inst);
    if (device >= 0 && argc > 4) {
        // One 1-spp frame per call, as PathTracingIntegrator::render (pt.cpp:90-99).
        for (uint32_t f = 0; f < frames; ++f) {
            if (vs_render(scene, f, 1, VS_FILM_FP32, nullptr) != VS_OK) {
                std::fprintf(stderr, "render: %s\n", vs_last_error(ctx));
                return 7;
            }
        }
        std::vector<float> rgba(static_cast<size_t>(info.width) * info.height * 4);
        if (vs_film_download(scene, rgba.data(), rgba.size() * sizeof(float), VS_FILM_LINEAR) != VS_OK) {
            std::fprintf(stderr, "download: %s\n", vs_last_error(ctx));
            return 8;
        }
        std::ofstream out(argv[4], std::ios::binary);
        out.write(reinterpret_cast<const char *>(rgba.data()), static_cast<std::streamsize>(rgba.size() * sizeof(float)));
    }
    vs_scene_destroy(scene);
    vs_context_destroy(ctx);
    return 0;
}
