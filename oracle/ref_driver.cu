// Test-infrastructure driver for the REFERENCE library (libflowfilter_gpu built
// from the reference sources by oracle/Makefile into oracle/_ref/).  It is
// never part of the product: it runs the reference's own stages and filters on
// inputs given as .npy files and writes their outputs as .npy files, so the
// CPU oracle and the golden fixtures can be pinned against the reference.
//
// Modes
//   norm   OUT.npy                     u8 -> normalised-float texture reads of 0..255
//   upmap  OUT.txt WMAX                nearest-texel index chosen by a normalised,
//                                      point-sampled, clamped texture at u = x/(W-1)
//                                      (the coarse-flow read of deltaFlowUpdate_k,
//                                      src/gpu/device/update_k.cu:151-155), listed
//                                      where it differs from floor(u*Wc)
//   stages IN_DIR OUT_DIR              every hot-path stage on the given inputs
//   wheelidx FLOWS.npy MAXFLOW OUT.npy  the reference's flowToColor_k (display_k.cu, compiled
//                                      into this driver from the reference sources) on the
//                                      given (H, W, 2) flows with an index-encoding wheel
//                                      (texel (i, j) = (j, i, 0, 255)) behind the texture
//                                      FlowToColor::configure sets up: OUT names the texel
//                                      each pixel read
//   lw FLOW.npy IMAGE.npy ITER OUT.npy  LaxWendroffPropagator(flow, image), setIterations(ITER)
//                                      unless ITER is 0, compute(): the propagated image
//   rotation IMAGE.npy FOCAL SH SW WX WY WZ ITER FLOW_OUT.npy PRED_OUT.npy
//                                      RotationalFlowImagePredictor(createPerspectiveCamera(
//                                      FOCAL, H, W, SH, SW), image), setAngularVelocity,
//                                      setIterations(ITER) unless 0, compute()
//   filter FRAMES.npy OUT.npy LEVELS MAXFLOW GAMMAS SMOOTHS DUMP [TIMING_CSV]
//                                      LEVELS=0: FlowFilter(h, w, S, maxflow, gamma)
//                                      LEVELS>=1: PyramidalFlowFilter(h, w, LEVELS)
//                                      GAMMAS / SMOOTHS are comma lists (level 0 first),
//                                      DUMP a comma list of frame indices to save.
//   filterpipe H W LEVELS MAXFLOW GAMMAS SMOOTHS
//                                      the same filters on frames read from stdin (H*W
//                                      uint8 each, until EOF); each frame's smoothed flow
//                                      (H*W*2 float32) is written to stdout
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cmath>
#include <string>
#include <vector>
#include <sstream>
#include <fstream>
#include <chrono>
#include <stdexcept>

#include <unistd.h>

#include <cuda_runtime.h>

#include "flowfilter/image.h"
#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/imagemodel.h"
#include "flowfilter/gpu/pyramid.h"
#include "flowfilter/gpu/propagation.h"
#include "flowfilter/gpu/update.h"
#include "flowfilter/gpu/flowsmoothing.h"
#include "flowfilter/gpu/flowfilter.h"
#include "flowfilter/gpu/camera.h"
#include "flowfilter/gpu/rotation.h"

// the reference's colour-lookup kernel, from its source tree (oracle/Makefile adds the
// reference's src/ directory to the include path)
#include "gpu/device/display_k.cu"

using namespace flowfilter;
using namespace flowfilter::gpu;

// ---------------------------------------------------------------- .npy io
struct Npy {
    std::string descr;          // '<f4', '|u1', '<i4'
    std::vector<size_t> shape;
    std::vector<char> data;
    size_t count() const { size_t n = 1; for (auto s : shape) n *= s; return n; }
};

static Npy npy_read(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    char magic[6];
    f.read(magic, 6);
    unsigned char ver[2];
    f.read((char*)ver, 2);
    uint32_t hlen = 0;
    if (ver[0] == 1) { uint16_t h16; f.read((char*)&h16, 2); hlen = h16; }
    else { f.read((char*)&hlen, 4); }
    std::string header(hlen, ' ');
    f.read(&header[0], hlen);
    Npy a;
    auto p = header.find("'descr':");
    auto q1 = header.find('\'', p + 8);
    auto q2 = header.find('\'', q1 + 1);
    a.descr = header.substr(q1 + 1, q2 - q1 - 1);
    if (header.find("'fortran_order': True") != std::string::npos)
        throw std::runtime_error("fortran order not supported: " + path);
    auto s1 = header.find('(', header.find("'shape':"));
    auto s2 = header.find(')', s1);
    std::stringstream ss(header.substr(s1 + 1, s2 - s1 - 1));
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        if (tok.find_first_not_of(" ") == std::string::npos) continue;
        a.shape.push_back(std::stoul(tok));
    }
    size_t item = (a.descr == "|u1") ? 1 : 4;
    a.data.resize(a.count() * item);
    f.read(a.data.data(), a.data.size());
    return a;
}

static void npy_write(const std::string& path, const std::string& descr,
                      const std::vector<size_t>& shape, const void* data, size_t bytes) {
    std::string sh = "(";
    for (size_t i = 0; i < shape.size(); ++i) sh += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    sh += ")";
    std::string header = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': " + sh + ", }";
    size_t total = 10 + header.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    header += std::string(pad, ' ') + "\n";
    std::ofstream f(path, std::ios::binary);
    f.write("\x93NUMPY", 6);
    char ver[2] = {1, 0};
    f.write(ver, 2);
    uint16_t hl = (uint16_t)header.size();
    f.write((char*)&hl, 2);
    f.write(header.data(), header.size());
    f.write((const char*)data, bytes);
}

static image_t wrap_host(void* data, int h, int w, int depth, int item) {
    image_t im;
    im.height = h; im.width = w; im.depth = depth;
    im.itemSize = item; im.pitch = (size_t)w * depth * item; im.data = data;
    return im;
}

static GPUImage upload_npy(const Npy& a, int depth) {
    int item = (a.descr == "|u1") ? 1 : 4;
    int h = (int)a.shape[0], w = (int)a.shape[1];
    GPUImage g(h, w, depth, item);
    image_t im = wrap_host((void*)a.data.data(), h, w, depth, item);
    g.upload(im);
    return g;
}

static void save_gpu(const std::string& path, GPUImage g) {
    int h = g.height(), w = g.width(), d = g.depth(), item = g.itemSize();
    std::vector<char> buf((size_t)h * w * d * item);
    image_t im = wrap_host(buf.data(), h, w, d, item);
    g.download(im);
    std::vector<size_t> shape = {(size_t)h, (size_t)w};
    if (d > 1) shape.push_back((size_t)d);
    npy_write(path, item == 1 ? "|u1" : "<f4", shape, buf.data(), buf.size());
}

// ---------------------------------------------------------------- probes
__global__ void probe_norm_k(cudaTextureObject_t tex, float* out) {
    int x = threadIdx.x;
    out[x] = tex2D<float>(tex, x, 0);
}

__global__ void probe_up_k(cudaTextureObject_t tex, int W, float* out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W) return;
    float u = (float)x / (float)(W - 1);
    float2 v = tex2D<float2>(tex, u, 0.0f);
    out[x] = v.x;
}

__global__ void probe_up_y_k(cudaTextureObject_t tex, int H, float* out) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= H) return;
    float v = (float)y / (float)(H - 1);
    float2 s = tex2D<float2>(tex, 0.0f, v);
    out[y] = s.y;
}

static int mode_norm(const std::string& out) {
    std::vector<unsigned char> v(256);
    for (int i = 0; i < 256; ++i) v[i] = (unsigned char)i;
    GPUImage g(1, 256, 1, 1);
    image_t im = wrap_host(v.data(), 1, 256, 1, 1);
    g.upload(im);
    GPUTexture tex(g, cudaChannelFormatKindUnsigned, cudaReadModeNormalizedFloat);
    float* d = nullptr;
    cudaMalloc(&d, 256 * sizeof(float));
    probe_norm_k<<<1, 256>>>(tex.getTextureObject(), d);
    std::vector<float> h(256);
    cudaMemcpy(h.data(), d, 256 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    npy_write(out, "<f4", {256}, h.data(), 256 * sizeof(float));
    return 0;
}

// Sweep: per (axis, W, Wc) the number of x where the texture's texel differs from
// floor(u*Wc); detail: full index arrays for the axis sizes the workloads use.
static void upmap_run(int dir, int W, int Wc, float* d, std::vector<float>& h) {
    int ch = dir == 0 ? 1 : Wc, cw = dir == 0 ? Wc : 1;
    std::vector<float> vals((size_t)ch * cw * 2);
    for (int i = 0; i < Wc; ++i) { vals[2 * i] = (float)i; vals[2 * i + 1] = (float)i; }
    GPUImage g(ch, cw, 2, 4);
    image_t im = wrap_host(vals.data(), ch, cw, 2, 4);
    g.upload(im);
    GPUTexture tex(g, cudaChannelFormatKindFloat, cudaAddressModeClamp,
                   cudaFilterModePoint, cudaReadModeElementType, true);
    if (dir == 0) probe_up_k<<<(W + 127) / 128, 128>>>(tex.getTextureObject(), W, d);
    else probe_up_y_k<<<(W + 127) / 128, 128>>>(tex.getTextureObject(), W, d);
    cudaMemcpy(h.data(), d, W * sizeof(float), cudaMemcpyDeviceToHost);
}

static int mode_upmap(const std::string& out, int wmax) {
    FILE* f = fopen(out.c_str(), "w");
    float* d = nullptr;
    const int cap = wmax > 4096 ? wmax : 4096;
    cudaMalloc(&d, (size_t)(cap + 8) * sizeof(float));
    std::vector<float> h(cap + 8);
    long mismatches = 0, checked = 0;
    for (int dir = 0; dir < 2; ++dir) {
        for (int W = 2; W <= wmax; ++W) {
            int cands[3] = {W / 2, (W + 1) / 2, W / 2 + 2};
            for (int ci = 0; ci < 3; ++ci) {
                int Wc = cands[ci];
                if (Wc < 1 || (ci > 0 && Wc == cands[ci - 1])) continue;
                upmap_run(dir, W, Wc, d, h);
                long cnt = 0; int first = -1;
                for (int x = 0; x < W; ++x) {
                    float u = (float)x / (float)(W - 1);
                    long m = (long)floorf(u * (float)Wc);
                    if (m < 0) m = 0;
                    if (m > Wc - 1) m = Wc - 1;
                    ++checked;
                    if ((long)h[x] != m) { ++cnt; if (first < 0) first = x; }
                }
                mismatches += cnt;
                if (cnt) fprintf(f, "%d %d %d %ld %d\n", dir, W, Wc, cnt, first);
            }
        }
    }
    fprintf(f, "# checked %ld mismatches %ld\n", checked, mismatches);
    fclose(f);
    // detail for the axis sizes of the workloads and the test cases
    const int pairs[][2] = {{2048, 1024}, {1024, 512}, {1088, 544}, {544, 272}, {640, 320}, {480, 240},
                            {320, 160}, {240, 120}, {1920, 960}, {960, 480}, {1080, 540}, {540, 270},
                            {1280, 640}, {720, 360}, {360, 180}, {256, 128}, {70, 35}, {53, 26},
                            {150, 75}, {75, 37}, {98, 49}, {49, 24}, {96, 48}, {64, 32}, {77, 38},
                            {61, 30}, {160, 80}, {120, 60}, {3, 1}, {2, 1}};
    const int np = sizeof(pairs) / sizeof(pairs[0]);
    std::vector<int> detail;
    for (int dir = 0; dir < 2; ++dir) {
        for (int k = 0; k < np; ++k) {
            int W = pairs[k][0], Wc = pairs[k][1];
            upmap_run(dir, W, Wc, d, h);
            detail.push_back(dir); detail.push_back(W); detail.push_back(Wc);
            for (int x = 0; x < W; ++x) detail.push_back((int)h[x]);
        }
    }
    npy_write(out + ".detail.npy", "<i4", {detail.size()}, detail.data(), detail.size() * sizeof(int));
    cudaFree(d);
    printf("upmap: checked %ld mismatches %ld\n", checked, mismatches);
    return 0;
}

// ---------------------------------------------------------------- stages
static int mode_stages(const std::string& in, const std::string& out) {
    Npy img8 = npy_read(in + "/img_u8.npy");
    Npy imgf = npy_read(in + "/img_f32.npy");
    Npy flow = npy_read(in + "/flow.npy");
    Npy scal = npy_read(in + "/scalar.npy");
    Npy vect = npy_read(in + "/vector.npy");
    Npy a0 = npy_read(in + "/a0.npy");
    Npy grad = npy_read(in + "/grad.npy");
    Npy a0old = npy_read(in + "/a0old.npy");
    Npy coarse = npy_read(in + "/coarse.npy");

    // image model, u8 and f32 input (src/gpu/imagemodel.cu:93-113)
    {
        GPUImage g = upload_npy(img8, 1);
        ImageModel m(g);
        m.compute();
        save_gpu(out + "/model_u8_a0.npy", m.getImageConstant());
        save_gpu(out + "/model_u8_grad.npy", m.getImageGradient());
        GPUImage gf = upload_npy(imgf, 1);
        ImageModel mf(gf);
        mf.compute();
        save_gpu(out + "/model_f32_a0.npy", mf.getImageConstant());
        save_gpu(out + "/model_f32_grad.npy", mf.getImageGradient());
    }
    // pyramid, 4 levels (src/gpu/pyramid.cu:110-167)
    {
        GPUImage g = upload_npy(img8, 1);
        ImagePyramid p(g, 4);
        p.compute();
        for (int l = 1; l < 4; ++l) save_gpu(out + "/pyr_u8_l" + std::to_string(l) + ".npy", p.getImage(l));
        GPUImage gf = upload_npy(imgf, 1);
        ImagePyramid pf(gf, 4);
        pf.compute();
        for (int l = 1; l < 4; ++l) save_gpu(out + "/pyr_f32_l" + std::to_string(l) + ".npy", pf.getImage(l));
    }
    // propagation (src/gpu/propagation.cu:80-134)
    const int borders[2] = {3, 0};
    for (int n = 1; n <= 4; ++n) {
        for (int b : borders) {
            GPUImage g = upload_npy(flow, 2);
            FlowPropagator pr(g, n);
            pr.setBorder(b);
            pr.compute();
            save_gpu(out + "/prop_n" + std::to_string(n) + "_b" + std::to_string(b) + ".npy", pr.getPropagatedFlow());
        }
    }
    // propagation with payload (src/gpu/propagation.cu:324-373)
    for (int n = 1; n <= 4; ++n) {
        GPUImage g = upload_npy(flow, 2);
        GPUImage s = upload_npy(scal, 1);
        GPUImage v = upload_npy(vect, 2);
        FlowPropagatorPayload pr(g, s, v, n);
        pr.compute();
        std::string tag = "/prop_payload_n" + std::to_string(n);
        save_gpu(out + tag + "_flow.npy", pr.getPropagatedFlow());
        save_gpu(out + tag + "_scalar.npy", pr.getPropagatedScalar());
        save_gpu(out + tag + "_vector.npy", pr.getPropagatedVector());
    }
    // update (src/gpu/update.cu:97-116); old image is the stage's own output buffer
    const float gammas[3] = {10.0f / (255.0f * 255.0f), 1.0f, 0.05f};
    const float maxflows[3] = {4.0f, 1.0f, 0.5f};
    for (int k = 0; k < 3; ++k) {
        GPUImage f = upload_npy(flow, 2);
        GPUImage ga0 = upload_npy(a0, 1);
        GPUImage gg = upload_npy(grad, 2);
        FlowUpdate up(f, ga0, gg, gammas[k], maxflows[k]);
        GPUImage old = up.getUpdatedImage();
        image_t im = wrap_host((void*)a0old.data.data(), (int)a0old.shape[0], (int)a0old.shape[1], 1, 4);
        old.upload(im);
        up.compute();
        save_gpu(out + "/update_k" + std::to_string(k) + "_flow.npy", up.getUpdatedFlow());
        save_gpu(out + "/update_k" + std::to_string(k) + "_image.npy", up.getUpdatedImage());
    }
    // delta update (src/gpu/update.cu:328-349)
    for (int k = 0; k < 3; ++k) {
        GPUImage c = upload_npy(coarse, 2);
        GPUImage d = upload_npy(vect, 2);
        GPUImage old = upload_npy(a0old, 1);
        GPUImage ga0 = upload_npy(a0, 1);
        GPUImage gg = upload_npy(grad, 2);
        DeltaFlowUpdate up(c, d, old, ga0, gg, gammas[k], maxflows[k]);
        up.compute();
        std::string tag = "/dupdate_k" + std::to_string(k);
        save_gpu(out + tag + "_flow.npy", up.getUpdatedFlow());
        save_gpu(out + tag + "_delta.npy", up.getUpdatedDeltaFlow());
        save_gpu(out + tag + "_image.npy", up.getUpdatedImage());
    }
    // smoothing (src/gpu/flowsmoothing.cu:74-108)
    for (int s = 1; s <= 3; ++s) {
        GPUImage g = upload_npy(flow, 2);
        FlowSmoother sm(g, s);
        sm.compute();
        save_gpu(out + "/smooth_s" + std::to_string(s) + ".npy", sm.getSmoothedFlow());
    }
    cudaError_t e = cudaDeviceSynchronize();
    printf("stages: %s\n", cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}

// ---------------------------------------------------------------- filters
static std::vector<float> parse_floats(const std::string& s) {
    std::vector<float> v; std::stringstream ss(s); std::string t;
    while (std::getline(ss, t, ',')) if (!t.empty()) v.push_back(std::stof(t));
    return v;
}
static std::vector<int> parse_ints(const std::string& s) {
    std::vector<int> v; std::stringstream ss(s); std::string t;
    while (std::getline(ss, t, ',')) if (!t.empty()) v.push_back(std::stoi(t));
    return v;
}

static int mode_filter(int argc, char** argv) {
    Npy frames = npy_read(argv[2]);
    std::string out = argv[3];
    int levels = atoi(argv[4]);
    float maxflow = (float)atof(argv[5]);
    std::vector<float> gammas = parse_floats(argv[6]);
    std::vector<int> smooths = parse_ints(argv[7]);
    std::vector<int> dump = parse_ints(argv[8]);
    std::string timing = argc > 9 ? argv[9] : "";
    int T = (int)frames.shape[0], H = (int)frames.shape[1], W = (int)frames.shape[2];
    size_t fsz = (size_t)H * W;

    std::vector<float> flows;
    std::vector<float> elapsed;
    std::vector<float> wall;
    std::vector<float> host(fsz * 2);
    image_t flowHost = wrap_host(host.data(), H, W, 2, 4);

    FlowFilter* ff = nullptr;
    PyramidalFlowFilter* pf = nullptr;
    if (levels == 0) {
        ff = new FlowFilter(H, W, smooths[0], maxflow, gammas[0]);
    } else {
        pf = new PyramidalFlowFilter(H, W, levels);
        pf->setGamma(gammas);
        pf->setSmoothIterations(smooths);
        pf->setMaxFlow(maxflow);
    }
    for (int t = 0; t < T; ++t) {
        image_t im = wrap_host(frames.data.data() + (size_t)t * fsz, H, W, 1, 1);
        auto t0 = std::chrono::high_resolution_clock::now();
        if (ff) { ff->loadImage(im); ff->compute(); elapsed.push_back(ff->elapsedTime()); }
        else { pf->loadImage(im); pf->compute(); elapsed.push_back(pf->elapsedTime()); }
        auto t1 = std::chrono::high_resolution_clock::now();
        wall.push_back(std::chrono::duration<float, std::milli>(t1 - t0).count());
        bool want = false;
        for (int d : dump) want |= (d == t);
        if (want) {
            if (ff) ff->downloadFlow(flowHost); else pf->downloadFlow(flowHost);
            flows.insert(flows.end(), host.begin(), host.end());
        }
    }
    npy_write(out, "<f4", {flows.size() / (fsz * 2), (size_t)H, (size_t)W, 2}, flows.data(), flows.size() * sizeof(float));
    if (!timing.empty()) {
        FILE* f = fopen(timing.c_str(), "w");
        fprintf(f, "frame,elapsed_ms,wall_ms\n");
        for (int t = 0; t < T; ++t) fprintf(f, "%d,%.6f,%.6f\n", t, elapsed[t], wall[t]);
        fclose(f);
    }
    delete ff;
    delete pf;
    cudaError_t e = cudaDeviceSynchronize();
    fprintf(stderr, "filter: %s\n", cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}

// Long sequences without files: frames (H*W uint8 each) arrive on stdin until EOF; after each
// frame the smoothed flow (H*W*2 float32, downloadFlow) goes to stdout.
static int mode_filterpipe(char** argv) {
    const int H = atoi(argv[2]), W = atoi(argv[3]), levels = atoi(argv[4]);
    const float maxflow = (float)atof(argv[5]);
    std::vector<float> gammas = parse_floats(argv[6]);
    std::vector<int> smooths = parse_ints(argv[7]);
    const size_t fsz = (size_t)H * W;
    std::vector<unsigned char> frame(fsz);
    std::vector<float> host(fsz * 2);
    image_t flowHost = wrap_host(host.data(), H, W, 2, 4);
    // the flows go to the original stdout; the library's own messages on stdout (the
    // filters print a line on their first frame) are sent to stderr instead
    fflush(stdout);
    const int data_fd = dup(1);
    if (data_fd < 0 || dup2(2, 1) < 0) { fprintf(stderr, "filterpipe: cannot redirect stdout\n"); return 1; }
    FILE* data = fdopen(data_fd, "wb");
    if (!data) { fprintf(stderr, "filterpipe: fdopen failed\n"); return 1; }
    FlowFilter* ff = nullptr;
    PyramidalFlowFilter* pf = nullptr;
    if (levels == 0) {
        ff = new FlowFilter(H, W, smooths[0], maxflow, gammas[0]);
    } else {
        pf = new PyramidalFlowFilter(H, W, levels);
        pf->setGamma(gammas);
        pf->setSmoothIterations(smooths);
        pf->setMaxFlow(maxflow);
    }
    int t = 0;
    while (fread(frame.data(), 1, fsz, stdin) == fsz) {
        image_t im = wrap_host(frame.data(), H, W, 1, 1);
        if (ff) { ff->loadImage(im); ff->compute(); ff->downloadFlow(flowHost); }
        else { pf->loadImage(im); pf->compute(); pf->downloadFlow(flowHost); }
        if (fwrite(host.data(), sizeof(float), fsz * 2, data) != fsz * 2) break;
        fflush(data);
        ++t;
    }
    fclose(data);
    delete ff;
    delete pf;
    cudaError_t e = cudaDeviceSynchronize();
    fprintf(stderr, "filterpipe: %d frames, %s\n", t, cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}

static int mode_wheelidx(const std::string& flows, float maxflow, const std::string& out) {
    Npy a = npy_read(flows);
    if (a.descr != "<f4" || a.shape.size() != 3 || a.shape[2] != 2)
        throw std::runtime_error("wheelidx: flows should be (H, W, 2) float32");
    const int h = (int)a.shape[0], w = (int)a.shape[1];
    GPUImage flow = upload_npy(a, 2);
    std::vector<unsigned char> wheel(256 * 256 * 4);
    for (int i = 0; i < 256; ++i)
        for (int j = 0; j < 256; ++j) {
            unsigned char* px = &wheel[4 * (i * 256 + j)];
            px[0] = (unsigned char)j;
            px[1] = (unsigned char)i;
            px[2] = 0;
            px[3] = 255;
        }
    GPUImage wimg(256, 256, 4, 1);
    image_t wi = wrap_host(wheel.data(), 256, 256, 4, 1);
    wimg.upload(wi);
    // the texture of FlowToColor::configure (display.cu:73-74)
    GPUTexture tex(wimg, cudaChannelFormatKindUnsigned, cudaReadModeElementType, true);
    GPUImage color(h, w, 4, 1);
    dim3 block(32, 32, 1), grid((w + 31) / 32, (h + 31) / 32, 1);
    flowToColor_k<<<grid, block>>>(flow.wrap<float2>(), tex.getTextureObject(), maxflow, color.wrap<uchar4>());
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) throw std::runtime_error(std::string("wheelidx: ") + cudaGetErrorString(e));
    save_gpu(out, color);
    return 0;
}

static GPUImage upload_image(const Npy& a) {
    if (a.descr != "<f4" || (a.shape.size() != 2 && !(a.shape.size() == 3 && a.shape[2] == 4)))
        throw std::runtime_error("image should be (H, W) or (H, W, 4) float32");
    return upload_npy(a, a.shape.size() == 2 ? 1 : 4);
}

static int mode_lw(const std::string& flowp, const std::string& imgp, int iters, const std::string& out) {
    GPUImage flow = upload_npy(npy_read(flowp), 2);
    GPUImage img = upload_image(npy_read(imgp));
    LaxWendroffPropagator lw(flow, img);
    if (iters > 0) lw.setIterations(iters);
    lw.compute();
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) throw std::runtime_error(std::string("lw: ") + cudaGetErrorString(e));
    save_gpu(out, lw.getPropagatedImage());
    return 0;
}

static int mode_rotation(char** argv) {
    GPUImage img = upload_image(npy_read(argv[2]));
    perspectiveCamera cam = createPerspectiveCamera((float)atof(argv[3]), img.height(), img.width(),
                                                    (float)atof(argv[4]), (float)atof(argv[5]));
    RotationalFlowImagePredictor pred(cam, img);
    pred.setAngularVelocity((float)atof(argv[6]), (float)atof(argv[7]), (float)atof(argv[8]));
    const int iters = atoi(argv[9]);
    if (iters > 0) pred.setIterations(iters);
    pred.compute();
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) throw std::runtime_error(std::string("rotation: ") + cudaGetErrorString(e));
    save_gpu(argv[10], pred.getOpticalFlow());
    save_gpu(argv[11], pred.getPredictedImage());
    const float cam4[4] = {cam.alphaX, cam.alphaY, cam.centerX, cam.centerY};
    std::vector<size_t> shape = {4};
    npy_write(std::string(argv[10]) + ".cam.npy", "<f4", shape, cam4, sizeof(cam4));
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: ref_driver MODE ...\n"); return 2; }
    std::string mode = argv[1];
    try {
        if (mode == "norm" && argc >= 3) return mode_norm(argv[2]);
        if (mode == "upmap" && argc >= 4) return mode_upmap(argv[2], atoi(argv[3]));
        if (mode == "stages" && argc >= 4) return mode_stages(argv[2], argv[3]);
        if (mode == "filter" && argc >= 9) return mode_filter(argc, argv);
        if (mode == "filterpipe" && argc >= 8) return mode_filterpipe(argv);
        if (mode == "lw" && argc >= 6) return mode_lw(argv[2], argv[3], atoi(argv[4]), argv[5]);
        if (mode == "rotation" && argc >= 12) return mode_rotation(argv);
        if (mode == "wheelidx" && argc >= 5) return mode_wheelidx(argv[2], (float)atof(argv[3]), argv[4]);
    } catch (const std::exception& e) {
        fprintf(stderr, "ref_driver: %s\n", e.what());
        return 3;
    }
    fprintf(stderr, "ref_driver: bad arguments for mode %s\n", mode.c_str());
    return 2;
}
