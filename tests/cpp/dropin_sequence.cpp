// Drives the C++ drop-in API (include/flowfilter/gpu/*.h) the way the reference's demos
// do, for tests/test_gpu_cpp_dropin.py.
//
//   dropin_sequence <frames.u8> <H> <W> <T> <levels> <out.f32> [<colour.u8>]
//
// levels 0: FlowFilter(H, W, 2, 4.0, 10.0); otherwise PyramidalFlowFilter(H, W, levels)
// with gamma[l] = 5 * 2^l, smoothIterations[l] = 1 + l % 3, maxflow 4.  Per frame the
// output holds downloadFlow (H*W*2), the getFlow() GPUImage taken once before the loop and
// downloaded after every compute (H*W*2), and downloadImage (H*W); after the last frame,
// an ImageModel of the last frame: constant (H*W) and gradient (H*W*2).  With a colour path,
// FlowToColor(filter.getFlow(), 4) after the last frame writes its RGBA image (H*W*4 bytes)
// there, as the reference's webcam demo builds it (demos/flowWebCam/src/flowWebCam.cpp:100).
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "flowfilter/colorwheel.h"
#include "flowfilter/gpu/display.h"
#include "flowfilter/gpu/flowfilter.h"
#include "flowfilter/gpu/imagemodel.h"

using namespace flowfilter;

static image_t host(void* data, int h, int w, int depth, int item) {
    image_t im;
    im.height = h;
    im.width = w;
    im.depth = depth;
    im.pitch = (size_t)w * depth * item;
    im.itemSize = item;
    im.data = data;
    return im;
}

template <typename F>
static bool throws(F&& f) {
    try {
        f();
    } catch (const std::exception&) {
        return true;
    }
    return false;
}

int main(int argc, char** argv) {
    if (argc != 7 && argc != 8) {
        std::fprintf(stderr, "usage: %s frames H W T levels out [colour]\n", argv[0]);
        return 2;
    }
    const int H = std::atoi(argv[2]), W = std::atoi(argv[3]), T = std::atoi(argv[4]), L = std::atoi(argv[5]);
    std::vector<unsigned char> frames((size_t)H * W * T);
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi || std::fread(frames.data(), 1, frames.size(), fi) != frames.size()) return 3;
    std::fclose(fi);
    FILE* fo = std::fopen(argv[6], "wb");
    if (!fo) return 4;

    std::vector<float> flow((size_t)H * W * 2), alias((size_t)H * W * 2), img((size_t)H * W);
    image_t flow_t = host(flow.data(), H, W, 2, 4), alias_t = host(alias.data(), H, W, 2, 4),
            img_t = host(img.data(), H, W, 1, 4);
    // FlowToColor of a filter's flow, and its error conventions
    auto colour = [&](gpu::GPUImage flowImg) -> int {
        if (argc != 8) return 0;
        gpu::FlowToColor c(flowImg, 4.0f);
        c.compute();
        std::vector<unsigned char> rgba((size_t)H * W * 4);
        image_t rgba_t = host(rgba.data(), H, W, 4, 1);
        c.downloadColorFlow(rgba_t);
        FILE* fc = std::fopen(argv[7], "wb");
        if (!fc || std::fwrite(rgba.data(), 1, rgba.size(), fc) != rgba.size()) return 11;
        std::fclose(fc);
        if (c.getMaxFlow() != 4.0f || !(c.elapsedTime() > 0.0f)) return 12;
        if (!throws([&] { c.setMaxFlow(0.0f); })) return 13;
        gpu::FlowToColor unset;
        if (!throws([&] { unset.compute(); }) || !throws([&] { unset.configure(); })) return 14;
        gpu::GPUImage one(H, W, 1, 4);
        if (!throws([&] { unset.setInputFlow(one); })) return 15;
        image_t wheel = getColorWheelRGBA();
        if (wheel.height != COLOR_WHEEL_HEIGHT || wheel.depth != 4 || wheel.data == nullptr) return 16;
        return 0;
    };
    auto dump = [&](gpu::GPUImage& a) {
        a.download(alias_t);
        std::fwrite(flow.data(), 4, flow.size(), fo);
        std::fwrite(alias.data(), 4, alias.size(), fo);
        std::fwrite(img.data(), 4, img.size(), fo);
    };
    try {
        if (L == 0) {
            gpu::FlowFilter f(H, W, 2, 4.0f, 10.0f);
            gpu::GPUImage a = f.getFlow();
            for (int t = 0; t < T; ++t) {
                image_t in = host(frames.data() + (size_t)t * H * W, H, W, 1, 1);
                f.loadImage(in);
                f.compute();
                f.downloadFlow(flow_t);
                f.downloadImage(img_t);
                dump(a);
            }
            if (f.getPropagationIterations() != 4 || f.getSmoothIterations() != 2 || f.height() != H) return 5;
            if (int rc = colour(f.getFlow())) return rc;
            if (!(f.elapsedTime() > 0.0f)) return 6;
        } else {
            gpu::PyramidalFlowFilter f(H, W, L);
            std::vector<float> g;
            std::vector<int> s;
            for (int l = 0; l < L; ++l) {
                g.push_back(5.0f * (float)(1 << l));
                s.push_back(1 + l % 3);
            }
            f.setGamma(g);
            f.setSmoothIterations(s);
            f.setMaxFlow(4.0f);
            gpu::GPUImage a = f.getFlow();
            for (int t = 0; t < T; ++t) {
                image_t in = host(frames.data() + (size_t)t * H * W, H, W, 1, 1);
                f.loadImage(in);
                f.compute();
                f.downloadFlow(flow_t);
                f.downloadImage(img_t);
                dump(a);
            }
            if (f.levels() != L || f.getSmoothIterations(L - 1) != s[L - 1]) return 5;
            if (int rc = colour(f.getFlow())) return rc;
            if (!(f.elapsedTime() > 0.0f)) return 6;
            // reference error conventions: bad level index, wrong vector size
            if (!throws([&] { f.setGamma(L, 1.0f); })) return 7;
            if (!throws([&] { f.setGamma(std::vector<float>(L + 1, 1.0f)); })) return 7;
        }
        // ImageModel over a GPUImage holding the last frame
        gpu::GPUImage dimg(H, W, 1, 1);
        image_t last = host(frames.data() + (size_t)(T - 1) * H * W, H, W, 1, 1);
        dimg.upload(last);
        gpu::ImageModel m(dimg);
        m.compute();
        std::vector<float> a0((size_t)H * W), grad((size_t)H * W * 2);
        image_t a0_t = host(a0.data(), H, W, 1, 4), grad_t = host(grad.data(), H, W, 2, 4);
        m.getImageConstant().download(a0_t);
        m.getImageGradient().download(grad_t);
        std::fwrite(a0.data(), 4, a0.size(), fo);
        std::fwrite(grad.data(), 4, grad.size(), fo);
        // constructor and shape errors
        if (!std::is_base_of<std::exception, std::invalid_argument>::value) return 8;
        bool bad_ctor = false;
        try {
            gpu::FlowFilter bad(0, W);
        } catch (const std::invalid_argument&) {
            bad_ctor = true;
        }
        if (!bad_ctor) return 8;
        image_t wrong = host(flow.data(), H + 1, W, 2, 4);
        if (!throws([&] { dimg.download(wrong); })) return 9;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 10;
    }
    std::fclose(fo);
    std::printf("ok\n");
    return 0;
}
