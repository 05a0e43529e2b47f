// Builds a pyramidal flow filter from the C++ drop-in stage classes (ImagePyramid,
// ImageModel, FlowPropagator, FlowPropagatorPayload, FlowUpdate, DeltaFlowUpdate,
// FlowSmoother) wired as the reference wires its FlowFilter, DeltaFlowFilter and
// PyramidalFlowFilter (src/gpu/flowfilter.cu:84-197, 371-503, 650-716), for
// tests/test_gpu_cpp_dropin.py.
//
//   dropin_stages <frames.u8> <H> <W> <T> <levels> <maxflow> <gammas> <smooths> <out.f32>
//
// gammas / smooths: comma lists, level 0 first; levels 0 = a single-level FlowFilter.  The
// output holds the smoothed level-0 flow (H*W*2 float) of every frame.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "flowfilter/gpu/flowsmoothing.h"
#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/imagemodel.h"
#include "flowfilter/gpu/propagation.h"
#include "flowfilter/gpu/pyramid.h"
#include "flowfilter/gpu/update.h"

using namespace flowfilter;
using namespace flowfilter::gpu;

template <typename T>
static std::vector<T> list(const char* s) {
    std::vector<T> v;
    std::stringstream ss(s);
    std::string t;
    while (std::getline(ss, t, ',')) v.push_back((T)std::atof(t.c_str()));
    return v;
}

// one level: FlowFilter (top) or DeltaFlowFilter (coarse != nullptr) built from stages
struct Level {
    bool top;
    ImageModel model;
    FlowUpdate update;
    DeltaFlowUpdate dupdate;
    FlowPropagator prop;
    FlowPropagatorPayload pprop;
    FlowSmoother smoother;
    bool first = true;

    Level(GPUImage image, GPUImage* coarse) : top(coarse == nullptr), model(image) {
        const int h = image.height(), w = image.width();
        if (top) {
            GPUImage dummy(h, w, 2, sizeof(float));
            update = FlowUpdate(dummy, model.getImageConstant(), model.getImageGradient(), 1.0f, 1.0f);
            smoother = FlowSmoother(update.getUpdatedFlow(), 1);
            prop = FlowPropagator(smoother.getSmoothedFlow(), 1);
            update.setInputFlow(prop.getPropagatedFlow());
        } else {
            GPUImage dd(h, w, 2, sizeof(float)), dold(h, w, 1, sizeof(float));
            dupdate = DeltaFlowUpdate(*coarse, dd, dold, model.getImageConstant(), model.getImageGradient());
            smoother = FlowSmoother(dupdate.getUpdatedFlow(), 1);
            pprop = FlowPropagatorPayload(smoother.getSmoothedFlow(), dupdate.getUpdatedImage(),
                                          dupdate.getUpdatedDeltaFlow());
            dupdate.setInputDeltaFlow(pprop.getPropagatedVector());
            dupdate.setInputImageOld(pprop.getPropagatedScalar());
        }
    }
    // the filters' setGamma (uint8 input: gamma / 255^2) and setMaxFlow (iterations = ceil)
    void params(float gamma, int smooth, float maxflow) {
        const float g = gamma / (255.0f * 255.0f);
        if (top) {
            update.setGamma(g);
            update.setMaxFlow(maxflow);
            prop.setIterations((int)std::ceil(maxflow));
        } else {
            dupdate.setGamma(g);
            dupdate.setMaxFlow(maxflow);
            pprop.setIterations((int)std::ceil(maxflow));
        }
        smoother.setIterations(smooth);
    }
    GPUImage flow() { return top ? update.getUpdatedFlow() : smoother.getSmoothedFlow(); }
    GPUImage updated_image() { return top ? update.getUpdatedImage() : dupdate.getUpdatedImage(); }
    void propagate() { top ? prop.compute() : pprop.compute(); }
    void compute_update() {
        if (first) {
            GPUImage a0 = model.getImageConstant();
            updated_image().copyFrom(a0);
            if (!top) pprop.getPropagatedScalar().copyFrom(a0);
            first = false;
        }
        top ? update.compute() : dupdate.compute();
        smoother.compute();
    }
    void compute_all() {  // FlowFilter::compute
        model.compute();
        if (first) {
            GPUImage a0 = model.getImageConstant();
            updated_image().copyFrom(a0);
            first = false;
        }
        propagate();
        top ? update.compute() : dupdate.compute();
        smoother.compute();
    }
};

int main(int argc, char** argv) {
    if (argc != 10) {
        std::fprintf(stderr, "usage: %s frames H W T levels maxflow gammas smooths out\n", argv[0]);
        return 2;
    }
    const int H = std::atoi(argv[2]), W = std::atoi(argv[3]), T = std::atoi(argv[4]);
    const int L = std::max(std::atoi(argv[5]), 1);
    const float maxflow = (float)std::atof(argv[6]);
    const std::vector<float> gammas = list<float>(argv[7]);
    const std::vector<int> smooths = list<int>(argv[8]);
    std::vector<unsigned char> frames((size_t)T * H * W);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(frames.data(), 1, frames.size(), f) != frames.size()) return 3;
    std::fclose(f);
    try {
        GPUImage input(H, W, 1, 1);
        ImagePyramid pyr(input, L);
        std::vector<std::unique_ptr<Level>> lv(L);
        lv[L - 1].reset(new Level(pyr.getImage(L - 1), nullptr));
        GPUImage coarse = lv[L - 1]->flow();
        for (int l = L - 2; l >= 0; --l) {
            lv[l].reset(new Level(pyr.getImage(l), &coarse));
            coarse = lv[l]->flow();
        }
        float m = maxflow;  // PyramidalFlowFilter::setMaxFlow: halved per level, top last
        for (int l = 0; l < L - 1; ++l) {
            lv[l]->params(gammas[l], smooths[l], m);
            m /= 2.0f;
        }
        lv[L - 1]->params(gammas[L - 1], smooths[L - 1], m);
        std::vector<float> out((size_t)H * W * 2);
        image_t ho;
        ho.height = H;
        ho.width = W;
        ho.depth = 2;
        ho.itemSize = 4;
        ho.pitch = (size_t)W * 8;
        ho.data = out.data();
        FILE* o = std::fopen(argv[9], "wb");
        for (int t = 0; t < T; ++t) {
            image_t hi;
            hi.height = H;
            hi.width = W;
            hi.depth = 1;
            hi.itemSize = 1;
            hi.pitch = (size_t)W;
            hi.data = frames.data() + (size_t)t * H * W;
            input.upload(hi);
            pyr.compute();
            if (L == 1) {
                lv[0]->compute_all();
            } else {  // PyramidalFlowFilter::compute
                lv[L - 1]->model.compute();
                lv[L - 1]->propagate();
                for (int l = 0; l < L - 1; ++l) {
                    lv[l]->model.compute();
                    lv[l]->propagate();
                }
                lv[L - 1]->compute_update();
                for (int l = 0; l < L - 1; ++l) lv[l]->compute_update();
            }
            lv[0]->smoother.getSmoothedFlow().download(ho);
            std::fwrite(out.data(), sizeof(float), out.size(), o);
        }
        std::fclose(o);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "dropin_stages: %s\n", e.what());
        return 1;
    }
    return 0;
}
