// Stage-1 net on one device image with no device allocation at all.
//
// Who needs this: callers that are not allowed to call cudaMalloc — plug-in hosts that account for
// every byte of device memory up front and hand a component only its input and output buffers, or
// processes whose device memory is already fully reserved by another framework's caching
// allocator, where an extra cudaMalloc would fail (or stall the device while memory is freed).
// The regular entry points allocate per-handle buffers; this one uses a fixed scratch array that is
// part of the library image instead.
//
// The scratch is a file-scope __device__ array: every GPU that loads the library holds it (9 MiB +
// 256 B) until the process exits. It holds the four L1 neighbour-sum planes of the image (up to
// kStaticS1Floats floats) after a reserved first 256 bytes; the level descriptor travels as a
// kernel parameter. Every call shares it, and it keeps the last call's contents; nothing in it has
// to start at zero, because each call writes every plane value it later reads. Calls that overlap
// on the GPU (different streams, or different host threads) race on the array.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>

#include "../../include/ccnn_inspect.h"
#include "kernels.h"
#include "model.h"

namespace ccnn {

void set_error(const std::string& msg);

namespace {

constexpr long long kStaticS1Floats = 2359296;  // 9 MiB of fp32: a 1920x1080 image needs 2,065,920
constexpr size_t kDescBytes = 256;  // reserved head of the array

static __device__ __align__(256) unsigned char g_stage1_scratch[kDescBytes + sizeof(float) * kStaticS1Floats];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};
std::map<std::string, Stage1W> g_weights;

// One-time set-up per device (with that device current): the device address of the array.
ccnn_status scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index out of range for the static scratch table");
        return CCNN_ERR_INVALID_ARG;
    }
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_stage1_scratch);
        if (e != cudaSuccess) {
            set_error(std::string("cudaGetSymbolAddress(static stage-1 scratch): ") + cudaGetErrorString(e));
            return CCNN_ERR_CUDA;
        }
        const cudaError_t e2 = stage1_setup();  // kernel attribute, no allocation
        if (e2 != cudaSuccess) {
            set_error(std::string("stage-1 kernel set-up: ") + cudaGetErrorString(e2));
            return CCNN_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return CCNN_OK;
}

ccnn_status stage1_weights(const char* model_path, Stage1W* w) {
    const std::string path = (model_path && model_path[0]) ? std::string(model_path) : bundled_model_dir() + "/cnn4face1_cntk.bin";
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_weights.find(path);
    if (it == g_weights.end()) {
        RawModel m;
        std::string err;
        Stage1W packed;
        if (!load_model_file(path, &m, &err) || !pack_model(m, 1, &packed, &err)) {
            set_error(err);
            return CCNN_ERR_MODEL;
        }
        if (m.min_w != kPatW || m.min_h != kPatH) {
            set_error("stage-1 model window is not 23x27");
            return CCNN_ERR_MODEL;
        }
        it = g_weights.emplace(path, packed).first;
    }
    *w = it->second;
    return CCNN_OK;
}

}  // namespace
}  // namespace ccnn

extern "C" CCNN_API ccnn_status ccnn_stage1_forward_static(const char* model_path, const float* d_img, int cols, int rows, size_t step,
                                                           float* d_resp, int resp_cap, int* resp_cols, int* resp_rows, void* stream) {
    using namespace ccnn;
    if (!d_img || !d_resp || !resp_cols || !resp_rows || (step % sizeof(float)) != 0 || step < sizeof(float) * (size_t)cols) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    if (cols < kPatW || rows < kPatH) {
        set_error("image smaller than the 23x27 stage-1 window");
        return CCNN_ERR_INVALID_ARG;
    }
    LevelDesc L{};
    L.w = cols;
    L.h = rows;
    L.mode = 0;
    L.scale = 1.f;
    L.inv_scale = 1.f;
    L.p1w = (cols - 3) >> 1;
    L.p1h = (rows - 3) >> 1;
    L.p2w = (L.p1w - 2) >> 1;
    L.p2h = (L.p1h - 2) >> 1;
    L.ow = L.p2w - 3;
    L.oh = L.p2h - 4;
    L.s1_pitch = (L.p1w + 31) / 32 * 32;
    L.s1_plane = (long long)L.s1_pitch * L.p1h;
    L.s1_off = 0;
    L.resp_off = 0;
    L.k1_tiles_x = (L.p1w + kK1TileX - 1) / kK1TileX;
    L.k2_tiles_x = (L.ow + kK2TileX - 1) / kK2TileX;
    L.k1_base = 0;
    L.k2_base = 0;
    L.img_off = 0;
    L.img_pitch = (int)(step / sizeof(float));
    L.img_vec = (L.img_pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(d_img) & 15) == 0) ? 1 : 0;
    *resp_cols = L.ow;
    *resp_rows = L.oh;
    if (4 * L.s1_plane > kStaticS1Floats) {
        set_error("image too large for the static scratch: its four L1 planes need " + std::to_string(4 * L.s1_plane) +
                  " floats, the maximum is 2359296 (about 1920x1080 or 2^21 pixels)");
        return CCNN_ERR_INVALID_ARG;
    }
    if ((long long)L.ow * L.oh > resp_cap) {
        set_error("response capacity too small");
        return CCNN_ERR_INVALID_ARG;
    }
    Stage1W w;
    ccnn_status st = stage1_weights(model_path, &w);
    if (st != CCNN_OK) return st;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    unsigned char* scratch = nullptr;
    st = scratch_address(dev, &scratch);
    if (st != CCNN_OK) return st;
    float* d_s1 = reinterpret_cast<float*>(scratch + kDescBytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = launch_stage1_front(w, &L, 1, d_img, d_s1, s);
    if (e == cudaSuccess) e = launch_stage1_back(w, &L, 1, d_s1, d_resp, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("static stage-1 forward: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}
