// Drives the drop-in camera, LaxWendroffPropagator and RotationalFlowImagePredictor classes
// (include/flowfilter/gpu/{camera,propagation,rotation}.h), for tests/test_gpu_cpp_dropin.py.
//
//   dropin_rotation <image.f32> <H> <W> <depth> <iterations> <out.f32>
//
// Camera createPerspectiveCamera(0.004, H, W, 0.003, 0.004), angular velocity
// (0.01, -0.02, 0.03).  Output: the camera (4 floats), the predictor's optical flow
// (H*W*2), its predicted image (H*W*depth), then a LaxWendroffPropagator of the same
// image along that flow with the same iterations (H*W*depth).
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "flowfilter/gpu/camera.h"
#include "flowfilter/gpu/propagation.h"
#include "flowfilter/gpu/rotation.h"

using namespace flowfilter;

static image_t host(void* data, int h, int w, int depth) {
    image_t im;
    im.height = h;
    im.width = w;
    im.depth = depth;
    im.pitch = (size_t)w * depth * 4;
    im.itemSize = 4;
    im.data = data;
    return im;
}

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s image H W depth iterations out\n", argv[0]);
        return 2;
    }
    const int H = std::atoi(argv[2]), W = std::atoi(argv[3]), D = std::atoi(argv[4]), N = std::atoi(argv[5]);
    std::vector<float> img((size_t)H * W * D);
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi || std::fread(img.data(), 4, img.size(), fi) != img.size()) return 3;
    std::fclose(fi);
    FILE* fo = std::fopen(argv[6], "wb");
    if (!fo) return 4;
    try {
        gpu::perspectiveCamera cam = gpu::createPerspectiveCamera(0.004f, H, W, 0.003f, 0.004f);
        std::fwrite(&cam, 4, 4, fo);
        gpu::GPUImage dimg(H, W, D, 4);
        image_t img_t = host(img.data(), H, W, D);
        dimg.upload(img_t);
        gpu::RotationalFlowImagePredictor pred(cam, dimg);
        pred.setAngularVelocity(0.01f, -0.02f, 0.03f);
        pred.setIterations(N);
        if (pred.getIterations() != N) return 5;
        pred.compute();
        std::vector<float> flow((size_t)H * W * 2), out((size_t)H * W * D);
        image_t flow_t = host(flow.data(), H, W, 2), out_t = host(out.data(), H, W, D);
        pred.getOpticalFlow().download(flow_t);
        pred.getPredictedImage().download(out_t);
        std::fwrite(flow.data(), 4, flow.size(), fo);
        std::fwrite(out.data(), 4, out.size(), fo);
        gpu::LaxWendroffPropagator lw(pred.getOpticalFlow(), dimg);
        lw.setIterations(N);
        lw.compute();
        if (!(lw.elapsedTime() > 0.0f) || lw.getDt() != 1.0f / float(N)) return 6;
        lw.getPropagatedImage().download(out_t);
        std::fwrite(out.data(), 4, out.size(), fo);
        // error conventions
        bool threw = false;
        try {
            lw.setIterations(0);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        if (!threw) return 7;
        threw = false;
        try {
            gpu::LaxWendroffPropagator bad;
            bad.compute();
        } catch (const std::logic_error&) {
            threw = true;
        }
        if (!threw) return 8;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 10;
    }
    std::fclose(fo);
    std::printf("ok\n");
    return 0;
}
